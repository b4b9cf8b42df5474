"""
Small utilities with the reference's names (pyrecon/utils.py): per-class loggers,
``distance``, ``broadcast_arrays``, ``setup_logging``.  They accept numpy arrays and
torch tensors alike.
"""
import sys
import time
import logging

import numpy as np

logger = logging.getLogger('pyrecon_b200')


def setup_logging(level=logging.INFO, stream=sys.stdout, filename=None, filemode='w', **kwargs):
    """Configure the root logger with elapsed-time prefixes (pyrecon/utils.py:26-70)."""
    if isinstance(level, str):
        level = {'info': logging.INFO, 'debug': logging.DEBUG, 'warning': logging.WARNING}[level.lower()]
    for handler in logging.root.handlers:
        logging.root.removeHandler(handler)
    t0 = time.time()

    class _Formatter(logging.Formatter):
        def format(self, record):
            self._style._fmt = '[%09.2f] ' % (time.time() - t0) + ' %(asctime)s %(name)-28s %(levelname)-8s %(message)s'
            return super(_Formatter, self).format(record)

    fmt = _Formatter(datefmt='%m-%d %H:%M ')
    handler = logging.FileHandler(filename, mode=filemode) if filename is not None else logging.StreamHandler(stream=stream)
    handler.setFormatter(fmt)
    logging.basicConfig(level=level, handlers=[handler], **kwargs)


class BaseMetaClass(type):
    """Gives every class a logger named after it and log_<level> class methods (pyrecon/utils.py:81-108)."""

    def __new__(meta, name, bases, class_dict):
        cls = super().__new__(meta, name, bases, class_dict)
        cls.logger = logging.getLogger(name)

        def make(level):
            @classmethod
            def log(cls, *args, **kwargs):
                getattr(cls.logger, level)(*args, **kwargs)
            return log

        for level in ['debug', 'info', 'warning', 'error', 'critical']:
            setattr(cls, 'log_{}'.format(level), make(level))
        return cls


class BaseClass(object, metaclass=BaseMetaClass):
    """Base class with shallow ``copy``."""

    def __copy__(self):
        new = self.__class__.__new__(self.__class__)
        new.__dict__.update(self.__dict__)
        return new

    def copy(self):
        return self.__copy__()


def broadcast_arrays(*arrays):
    """N 1D arrays -> N arrays of shape (n1, 1, ...), (1, n2, ...), ... (pyrecon/utils.py:125-143)."""
    out = []
    for iaxis, array in enumerate(arrays):
        sl = [None] * len(arrays)
        sl[iaxis] = slice(None)
        out.append(array[tuple(sl)])
    return tuple(out)


def distance(position):
    """Cartesian distance along the last axis (pyrecon/utils.py:146-148)."""
    try:
        import torch
        if isinstance(position, torch.Tensor):
            return torch.sqrt((position ** 2).sum(dim=-1))
    except ImportError:
        pass
    return np.sqrt((position ** 2).sum(axis=-1))
