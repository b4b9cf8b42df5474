"""``python -m pyrecon_b200 config.yaml``: standalone reconstruction (see pyrecon_b200.cli)."""
import sys

from .cli import main

sys.exit(main())
