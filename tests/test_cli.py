"""
The standalone entry point (pyrecon_b200.cli, the reference's bin/pyrecon): configuration handling,
catalogue I/O and the redshift-distance relation on the CPU; a full run on the GPU against the API.
"""
import os

import numpy as np
import pytest

from pyrecon_b200 import cli


def test_config_defaults_file_and_errors(tmp_path):
    fn = str(tmp_path / 'config.yaml')
    with open(fn, 'w') as file:
        file.write('input:\n  data_fn: d.npz\n  xyz: Position\nmesh:\n  nmesh: 64\ncosmology:\n  f: 0.8\n  bias: 2.\n')
    config = cli.load_config(fn)
    assert config['algorithm'] == {'name': 'MultiGridReconstruction', 'convention': 'RecSym'}
    assert config['mesh'] == {'nmesh': 64, 'dtype': 'f4'}
    assert config['delta'] == {'smoothing_radius': 15.}
    assert config['input']['xyz'] == 'Position'
    bad = cli.load_config(fn, algorithm={'convention': 'nope'})
    with pytest.raises(cli.ConfigError):
        cli.run(bad)
    nodata = cli.load_config(None)
    with pytest.raises(cli.ConfigError):
        cli.run(nodata)


@pytest.mark.parametrize('ext', ['.npz', '.npy', '.parquet', '.feather', '.fits'])
def test_catalogue_io_roundtrip(tmp_path, ext):
    rng = np.random.default_rng(0)
    catalog = {'Position': rng.normal(size=(50, 3)), 'RA': rng.uniform(0, 360, 50).astype('f4'),
               'Weight': rng.uniform(size=50)}
    fn = str(tmp_path / ('cat' + ext))
    cli.write_columns(fn, catalog)
    back = cli.read_columns(fn, ['Position', 'Weight', 'RA'])
    for k, v in catalog.items():
        assert back[k].dtype == v.dtype
        np.testing.assert_array_equal(back[k], v)
    with pytest.raises(cli.ConfigError):
        cli.read_columns(str(tmp_path / 'cat.txt'), ['RA'])


def test_comoving_distance_flat_lcdm():
    """Flat LambdaCDM, Omega_m = 0.3: comoving distance to z = 1 is 2312.7 Mpc/h (3303.8 Mpc at h = 0.7);
    monotonic, zero at z = 0, and inverted by DistanceToRedshift."""
    from pyrecon_b200 import utils
    dist = cli.comoving_distance_function(0.3)
    z = np.array([0., 0.5, 1., 2.])
    d = dist(z)
    assert d[0] == 0. and np.all(np.diff(d) > 0)
    assert abs(d[2] - 2312.7) < 0.5
    zz = utils.DistanceToRedshift(dist, zmax=10., nz=512)(d[1:])
    np.testing.assert_allclose(zz, z[1:], rtol=1e-6)


def test_mask_and_weight_expressions():
    expr, cols = cli._decode_eval('${Z} > 0.4 & (${W} < 2)')
    assert expr == 'Z > 0.4 & (W < 2)' and cols == ['Z', 'W']
    assert cli.sepjoin('/a/', '/b') == '/b' and cli.sepjoin('a', 'b') == '/a/b'


@pytest.mark.gpu
@pytest.mark.parametrize('convention,ext', [('RecSym', '.npz'), ('RecIso', '.npz'), ('RSD', '.npz'),
                                            ('RecSym', '.fits')])
def test_cli_run_equals_api(tmp_path, convention, ext):
    """A configuration run (xyz catalogues in .npz or FITS, mask and weight expressions, randoms selection
    function) writes the shifted positions the API gives for the same inputs."""
    import pyrecon_b200
    from pyrecon_b200 import mocks
    data = mocks.lognormal_positions_numpy(20000, 32, 1000., 2000., seed=1, field_seed=2)
    randoms = mocks.uniform_positions_numpy(60000, 1000., 2000., seed=3)
    w = np.random.default_rng(4).uniform(0.5, 1.5, len(data))
    cli.write_columns(str(tmp_path / ('data' + ext)), {'Position': data, 'W': w})
    cli.write_columns(str(tmp_path / ('randoms' + ext)), {'Position': randoms})
    config = cli.load_config(None, input={'dir': str(tmp_path), 'data_fn': 'data' + ext, 'randoms_fn': 'randoms' + ext,
                                          'xyz': 'Position', 'weights_data': '${W}', 'mask_data': '${W} > 0.6'},
                             output={'dir': str(tmp_path), 'data_fn': 'out_data' + ext,
                                     'randoms_fn': 'out_randoms' + ext, 'xyz_rec': 'Position_rec',
                                     'columns_data': ['W']},
                             algorithm={'name': 'MultiGridReconstruction', 'convention': convention},
                             cosmology={'f': 0.8, 'bias': 2.}, mesh={'nmesh': 32, 'boxpad': 1.5, 'dtype': 'f8'})
    cli.run(config)
    out_d = cli.read_columns(str(tmp_path / ('out_data' + ext)), ['Position_rec', 'W'])
    out_r = cli.read_columns(str(tmp_path / ('out_randoms' + ext)), ['Position_rec'])
    keep = w > 0.6
    rec = pyrecon_b200.MultiGridReconstruction(f=0.8, bias=2., nmesh=32, boxpad=1.5, dtype='f8', positions=randoms)
    rec.assign_data(data[keep], w[keep])
    rec.assign_randoms(randoms)
    rec.set_density_contrast(smoothing_radius=15.)
    rec.run()
    field = 'rsd' if convention == 'RSD' else 'disp+rsd'
    np.testing.assert_array_equal(out_d['Position_rec'], rec.read_shifted_positions(data[keep], field=field))
    np.testing.assert_array_equal(out_d['W'], w[keep])
    ref_r = randoms if convention == 'RSD' else \
        rec.read_shifted_positions(randoms, field='disp+rsd' if convention == 'RecSym' else 'disp')
    np.testing.assert_array_equal(out_r['Position_rec'], ref_r)
