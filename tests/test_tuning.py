"""
The autotuner's wisdom (pyrecon_b200.tuning): JSON round trip and the tuning table on the host (CPU),
tuning a mesh on the device and reusing the saved wisdom through the reconstruction classes' own
fft_wisdom / save_fft_wisdom arguments (GPU).
"""
import json

import numpy as np
import pytest


def test_wisdom_roundtrip_and_table(tmp_path):
    from pyrecon_b200 import tuning, _lib
    w = tuning.Wisdom({'NVIDIA B200': {'mg_jacobi': {'512': 32, 256: 16}}})
    path = str(tmp_path / 'w.json')
    w.save(path)
    data = json.load(open(path))
    assert data['format'] == tuning.FORMAT and data['devices']['NVIDIA B200']['mg_jacobi'] == {'256': 16, '512': 32}
    w2 = tuning.Wisdom.load(path)
    assert w2.entries == {'NVIDIA B200': {'mg_jacobi': {512: 32, 256: 16}}}
    assert w2.covers('NVIDIA B200', (512, 512, 512), 'f4') is False      # levels 128 .. 4 missing
    w2.update('NVIDIA B200', {'mg_jacobi': {n: 0 for n in [128, 64, 32, 16, 8, 4]}})
    assert w2.covers('NVIDIA B200', (512, 512, 512), 'f4')
    assert not w2.covers('NVIDIA B200', (512, 512, 512), 'f8')
    assert not w2.covers('other', (512, 512, 512), 'f4')
    try:
        assert w2.apply('NVIDIA B200') == 8
        assert _lib.tune_get('mg_jacobi', 512) == 32 and _lib.tune_get('mg_jacobi', 8) == 0
        assert _lib.tune_get('mg_jacobi', 1000, -7) == -7
    finally:
        _lib.tune_clear()
    assert _lib.tune_get('mg_jacobi', 512) == -1
    with pytest.raises(ValueError):
        open(str(tmp_path / 'bad.json'), 'w').write('{"format": "other"}')
        tuning.Wisdom.load(str(tmp_path / 'bad.json'))


def test_mg_levels():
    from pyrecon_b200 import tuning
    assert tuning.mg_levels((512, 512, 512))[-1] == (4, 4, 4)
    assert tuning.mg_levels((384, 384, 384))[-1] == (3, 3, 3)
    assert tuning.mg_levels((13, 11, 9)) == [(13, 11, 9)]


@pytest.mark.gpu
def test_autotune_and_reuse(tmp_path):
    """Tuning a 64^3 mesh times every candidate per level; the reconstruction built with save_fft_wisdom
    writes the wisdom file, a second one built with fft_wisdom applies it without timing, and the shifted
    positions are identical either way (two sweeps per pass give the bits of one)."""
    import pyrecon_b200
    from pyrecon_b200 import tuning, _lib
    best, timings = tuning.autotune((64, 64, 64), 'f4', repeats=2)
    assert set(best['mg_jacobi']) == {64, 32, 16, 8, 4}
    for n, ms in timings['mg_jacobi'].items():
        assert best['mg_jacobi'][n] == min(ms, key=ms.get) and all(t > 0 for t in ms.values())
    rng = np.random.default_rng(3)
    data = (2000. + rng.uniform(-400., 400., (20000, 3))).astype('f4')
    randoms = (2000. + rng.uniform(-400., 400., (60000, 3))).astype('f4')
    out = {}
    path = str(tmp_path / 'wisdom.json')
    try:
        for kind, kw in [('plain', {}), ('tuned', dict(save_fft_wisdom=path)), ('reused', dict(fft_wisdom=path))]:
            if kind == 'reused':
                _lib.tune_clear()
            rec = pyrecon_b200.MultiGridReconstruction(f=0.8, bias=2., nmesh=64, boxsize=1000., boxcenter=2000.,
                                                       dtype='f4', **kw)
            if kind != 'plain':
                assert rec.fft_wisdom is not None and rec.fft_wisdom.covers(tuning.device_name(), (64,) * 3, 'f4')
                assert _lib.tune_get('mg_jacobi', 64) >= 0
            rec.assign_data(data)
            rec.assign_randoms(randoms)
            rec.set_density_contrast(smoothing_radius=15.)
            rec.run()
            out[kind] = rec.read_shifted_positions(data)
    finally:
        _lib.tune_clear()
    assert np.array_equal(out['plain'], out['tuned']) and np.array_equal(out['plain'], out['reused'])
