"""
Standalone reconstruction from a YAML configuration (the reference's ``bin/pyrecon`` entry point,
pyrecon bin/pyrecon:70-423), on CUDA:

    python -m pyrecon_b200 config.yaml [--data-fn ...] [--randoms-fn ...] [--output-data-fn ...]
                                        [--output-randoms-fn ...] [--growth-rate F] [--galaxy-bias B]

Configuration sections as in the reference: ``input`` (data_fn, randoms_fn, dir, xyz / rdz
columns, optionally per catalogue as xyz_data, rdz_randoms..., weights / mask expressions with
${column} references, hdf5_prefix), ``output`` (data_fn, randoms_fn, dir, columns to keep, xyz / rdz /
xyz_rec / rdz_rec columns), ``algorithm`` (name, convention RecSym / RecIso / RSD, los, and the
keywords of ``run``), ``delta`` (set_density_contrast keywords, selection_function uniform /
randoms), ``cosmology`` (f, bias, Omega_m for rdz conversions), ``mesh`` (nmesh, dtype, boxsize,
cellsize, boxpad, wrap...).

Catalogue formats, by extension: FITS (.fits: fitsio when installed, else the built-in binary-table
reader / writer of :mod:`pyrecon_b200.fits`), HDF5 (.hdf5, .h5, ..., needs h5py),
numpy (.npz: one array per column, .npy: a structured array) and Arrow (.parquet, .feather, needs
pyarrow).  Redshift <-> comoving distance (Mpc/h) of a flat LambdaCDM model with Omega_m: astropy's
when it is installed, else the same integral computed here.
"""
import os
import re
import sys
import logging
import argparse
from numbers import Number

import numpy as np

from . import utils


class ConfigError(Exception):
    """A configuration that cannot be run."""


EXTENSIONS = {'fits': ['.fits'], 'hdf5': ['.hdf', '.h4', '.hdf4', '.he2', '.h5', '.hdf5', '.he5', '.h5py'],
              'npz': ['.npz'], 'npy': ['.npy'], 'parquet': ['.parquet'], 'feather': ['.feather', '.arrow']}


def _format_of(fn):
    for fmt, exts in EXTENSIONS.items():
        if any(fn.endswith(ext) for ext in exts):
            return fmt
    allowed = ', '.join('{} ({})'.format(fmt, exts) for fmt, exts in EXTENSIONS.items())
    raise ConfigError('File format of {} is not recognized. Formats {} only are handled.'.format(fn, allowed))


def sepjoin(*paths):
    """Join HDF5 dataset paths with single '/' separators (an absolute later path restarts)."""
    sep, out = '/', ''
    for path in paths:
        if path is None:
            continue
        if out.endswith(sep) and path.startswith(sep):
            out = path
        elif not out.endswith(sep) and not path.startswith(sep):
            out += sep + path
        else:
            out += path
    return out


def read_columns(fn, columns, hdf5_prefix=''):
    """The requested columns of a catalogue file, as a dict of numpy arrays."""
    fmt = _format_of(fn)
    if fmt == 'fits':
        try:
            import fitsio
        except ImportError:        # the built-in binary-table reader
            from . import fits
            return fits.read(fn, columns=columns)
        tmp = fitsio.read(fn, columns=columns)
        return {col: tmp[col] for col in columns}
    if fmt == 'hdf5':
        import h5py
        with h5py.File(fn, 'r') as file:
            return {col: file[sepjoin(hdf5_prefix, col)][:] for col in columns}
    if fmt == 'npz':
        with np.load(fn) as z:
            return {col: z[col] for col in columns}
    if fmt == 'npy':
        arr = np.load(fn)
        return {col: arr[col] for col in columns}
    import pyarrow.feather
    import pyarrow.parquet
    table = pyarrow.parquet.read_table(fn, columns=columns) if fmt == 'parquet' else \
        pyarrow.feather.read_table(fn, columns=columns)
    return {col: _arrow_column(table.column(col)) for col in columns}


def _arrow_column(col):
    arr = col.to_numpy()
    if arr.dtype == object:                 # fixed-size lists (e.g. positions of shape (N, 3))
        arr = np.stack(arr)
    return arr


def write_columns(fn, catalog, hdf5_prefix=''):
    """Write a dict of columns (first axis: rows) to a catalogue file."""
    fmt = _format_of(fn)
    columns = list(catalog.keys())
    if fmt == 'fits':
        array = np.empty(len(catalog[columns[0]]), dtype=[(c, catalog[c].dtype, catalog[c].shape[1:]) for c in columns])
        for c in columns:
            array[c] = catalog[c]
        try:
            import fitsio
        except ImportError:        # the built-in binary-table writer
            from . import fits
            fits.write(fn, array)
        else:
            fitsio.write(fn, array, clobber=True)
    elif fmt == 'hdf5':
        import h5py
        with h5py.File(fn, 'w') as file:
            for c in columns:
                file[sepjoin(hdf5_prefix, c)] = catalog[c]
    elif fmt == 'npz':
        np.savez(fn, **catalog)
    elif fmt == 'npy':
        array = np.empty(len(catalog[columns[0]]), dtype=[(c, catalog[c].dtype, catalog[c].shape[1:]) for c in columns])
        for c in columns:
            array[c] = catalog[c]
        np.save(fn, array)
    else:
        import pyarrow
        import pyarrow.feather
        import pyarrow.parquet
        data = {}
        for c in columns:
            v = catalog[c]
            data[c] = pyarrow.array(list(v)) if v.ndim > 1 else pyarrow.array(v)
        table = pyarrow.table(data)
        if fmt == 'parquet':
            pyarrow.parquet.write_table(table, fn)
        else:
            pyarrow.feather.write_feather(table, fn)


def comoving_distance_function(omega_m):
    """z -> comoving distance in Mpc/h of a flat LambdaCDM model (no radiation), as the reference gets it
    from astropy's FlatLambdaCDM(H0=70, Om0=omega_m) times h."""
    try:
        from astropy.cosmology import FlatLambdaCDM
    except ImportError:
        FlatLambdaCDM = None
    if FlatLambdaCDM is not None:
        cosmo = FlatLambdaCDM(H0=70, Om0=omega_m)
        return lambda z: cosmo.comoving_distance(z).value * cosmo.h
    from scipy import integrate
    hubble_distance = 299792.458 / 100.                 # c / (100 km/s/Mpc), Mpc/h

    def inverse_e(z):
        return 1. / np.sqrt(omega_m * (1. + z) ** 3 + 1. - omega_m)

    def comoving_distance(z):
        z = np.asarray(z, dtype='f8')
        flat = z.ravel()
        order = np.argsort(flat)
        out = np.empty_like(flat)
        prev_z, prev_d = 0., 0.
        for i in order:                                   # cumulative integral over sorted redshifts
            zi = flat[i]
            prev_d += integrate.quad(inverse_e, prev_z, zi, epsabs=0., epsrel=1e-12, limit=200)[0]
            prev_z = zi
            out[i] = prev_d
        return (hubble_distance * out).reshape(z.shape)

    return comoving_distance


def _make_list(cols):
    if cols is None:
        return []
    return [cols] if isinstance(cols, str) else list(cols)


def _unique(cols):
    out = []
    for c in cols:
        if c not in out:
            out.append(c)
    return out


def _decode_eval(s):
    """'${a} * ${b}' -> ('a * b', ['a', 'b'])."""
    if s is None:
        return '', []
    out, columns = str(s), []
    for m in re.finditer(r'(\${.*?})', str(s)):
        col = m.group(1)[2:-1]
        out = out.replace(m.group(1), col)
        if col not in columns:
            columns.append(col)
    return out, columns


def load_config(config_fn=None, **input_config):
    """The reference's defaults, updated by ``input_config`` then by the YAML file."""
    import yaml
    config = {'input': {}, 'output': {}, 'algorithm': {'name': 'MultiGridReconstruction', 'convention': 'RecSym'},
              'delta': {'smoothing_radius': 15.}, 'cosmology': {}, 'mesh': {'nmesh': 512, 'dtype': 'f4'}}

    def update(c1, c2):
        for section, value in c2.items():
            c1.setdefault(section, {})
            c1[section].update(value or {})
        for section in c1:
            for name, value in c1[section].items():
                if not isinstance(value, Number) and not value:
                    c1[section][name] = None

    update(config, input_config)
    if config_fn is not None:
        with open(config_fn, 'r') as file:
            update(config, yaml.safe_load(file) or {})
    return config


def run(config, device=None):
    """Run the reconstruction described by ``config`` (load_config); returns {name: catalogue dict} of the
    catalogues written (also those without an output file are not returned)."""
    import pyrecon_b200
    logger = logging.getLogger('Main')
    config = {k: dict(v) for k, v in config.items()}
    Algorithm = getattr(pyrecon_b200, config['algorithm'].pop('name'))
    cosmo = {k: v for k, v in config['cosmology'].items() if k in ['f', 'bias']}
    cosmo['los'] = config['algorithm'].pop('los', None)
    convention = str(config['algorithm'].pop('convention')).lower()
    config['algorithm'].pop('nthreads', None)
    if convention not in ['recsym', 'reciso', 'rsd']:
        raise ConfigError('Unknown convention {}. Choices are {}'.format(convention, ['recsym', 'reciso', 'rsd']))
    logger.info('Convention is {}.'.format(convention))

    def distance_fn():
        omega_m = config['cosmology'].get('Omega_m', None)
        if omega_m is None:
            raise ConfigError('Provide Omega_m for redshift -> distance conversion.')
        return comoving_distance_function(omega_m)

    selection = (config['delta'].pop('selection_function', '') or '').lower()
    if selection not in ['uniform', 'randoms', '']:
        raise ConfigError('Unknown input selection function {}. Choices are {}'.format(selection,
                                                                                       ['uniform', 'randoms', '']))
    input_fns, output_fns = {}, {}
    for name in ['data', 'randoms']:
        fn = config['input'].get('{}_fn'.format(name), None)
        if fn is None:
            if name == 'data':
                raise ConfigError('Please provide data catalog.')
            if selection == 'randoms':
                raise ConfigError('Please provide randoms catalog.')
            if not selection:
                logger.info('No randoms provided.')
                selection = 'uniform'
        else:
            input_fns[name] = fn
        fn = config['output'].get('{}_fn'.format(name), None)
        if fn is not None:
            if name not in input_fns:
                raise ConfigError('Cannot output {} catalog if not provided as input.'.format(name))
            output_fns[name] = fn
    if not selection:
        selection = 'randoms'
    logger.info('Using {} selection function.'.format(selection))

    formats = ['rdz', 'xyz']
    catalogs, positions, weights, keep = {}, {}, {}, {}
    for name in input_fns:
        # per-catalogue format (xyz_data, rdz_randoms, ...) first, then the common one (xyz, rdz)
        fmt, position_columns = None, None
        for keys in [['{}_{}'.format(f, name) for f in formats], formats]:
            for f, key in zip(formats, keys):
                cols = config['input'].get(key, None)
                if cols is not None:
                    if fmt is not None:
                        raise ConfigError('Cannot use two different input formats')
                    fmt, position_columns = f, cols
            if fmt is not None:
                break
        if fmt is None:
            raise ConfigError('Unknown input format. Choices are {}'.format(formats))
        position_columns = _make_list(position_columns)
        fn = os.path.join(config['input'].get('dir', '') or '', input_fns[name])
        mask_str, mask_columns = _decode_eval(config['input'].get('mask_{}'.format(name), config['input'].get('mask')))
        weight_str, weight_columns = _decode_eval(config['input'].get('weights_{}'.format(name),
                                                                      config['input'].get('weights')))
        keep[name] = _make_list(config['output'].get('columns_{}'.format(name), config['output'].get('columns')))
        columns = _unique(position_columns + weight_columns + mask_columns + keep[name])
        logger.info('Loading {} catalog {}.'.format(name, fn))
        catalog = read_columns(fn, columns, hdf5_prefix=config['input'].get('hdf5_prefix', '') or '')
        logger.info('Size of catalog {} is {:d}.'.format(name, len(catalog[columns[0]])))
        if mask_str:
            mask = eval(mask_str, dict(np=np, **catalog), {})
            catalog = {c: v[mask] for c, v in catalog.items()}
            logger.info('Size of catalog {} after masking is {:d}.'.format(name, len(catalog[columns[0]])))
        if fmt == 'rdz':
            if len(position_columns) != 3:
                raise ConfigError('Format rdz requires 3 position columns')
            dist = distance_fn()(catalog[position_columns[2]])
            positions[name] = utils.sky_to_cartesian(dist, catalog[position_columns[0]], catalog[position_columns[1]])
        elif len(position_columns) == 3:
            positions[name] = np.array([catalog[c] for c in position_columns]).T
        elif len(position_columns) == 1:
            positions[name] = catalog[position_columns[0]]
        else:
            raise ConfigError('Format xyz requires 1 or 3 position columns')
        weights[name] = eval(weight_str, dict(np=np, **catalog), {}) if weight_str else None
        catalogs[name] = {c: v for c, v in catalog.items() if c in keep[name]}

    recon = Algorithm(device=device, **cosmo, **config['mesh'],
                      positions=positions['randoms'] if selection == 'randoms' else None)
    recon.assign_data(positions['data'], weights['data'])
    if selection == 'randoms':
        recon.assign_randoms(positions['randoms'], weights['randoms'])
    recon.set_density_contrast(**config['delta'])
    recon.run(**config['algorithm'])

    rec = {}
    field = 'rsd' if convention == 'rsd' else 'disp+rsd'
    if isinstance(recon, pyrecon_b200.OriginalIterativeFFTParticleReconstruction):
        rec['data'] = recon.read_shifted_positions('data', field=field)
    else:
        rec['data'] = recon.read_shifted_positions(positions['data'], field=field)
    if 'randoms' in output_fns:
        if convention == 'rsd':
            rec['randoms'] = positions['randoms']             # RSD removal only: randoms unchanged
        else:
            rec['randoms'] = recon.read_shifted_positions(positions['randoms'],
                                                          field='disp+rsd' if convention == 'recsym' else 'disp')
    written = {}
    for name in output_fns:
        catalog = dict(catalogs[name])
        for tag, pos in zip(['', '_rec'], [positions[name], rec[name]]):
            for f in formats:
                cols = config['output'].get('{}{}_{}'.format(f, tag, name), None)
                if cols is None:
                    cols = config['output'].get('{}{}'.format(f, tag), None)
                if cols is None:
                    continue
                cols = _make_list(cols)
                if f == 'rdz':
                    if len(cols) != 3:
                        raise ConfigError('Format rdz requires 3 position columns')
                    dist, ra, dec = utils.cartesian_to_sky(pos)
                    z = utils.DistanceToRedshift(distance_fn())(dist)
                    for c, v in zip(cols, [ra, dec, z]):
                        catalog[c] = v
                elif len(cols) == 3:
                    for i, c in enumerate(cols):
                        catalog[c] = pos[:, i]
                elif len(cols) == 1:
                    catalog[cols[0]] = pos
                else:
                    raise ConfigError('Format xyz requires 1 or 3 position columns')
        fn = os.path.join(config['output'].get('dir', '') or '', output_fns[name])
        logger.info('Saving {} catalog to {}.'.format(name, fn))
        utils.mkdir(os.path.dirname(fn) or '.')
        write_columns(fn, catalog, hdf5_prefix=config['output'].get('hdf5_prefix', '') or '')
        written[name] = catalog
    return written


def main(args=None, **input_config):
    parser = argparse.ArgumentParser(formatter_class=argparse.ArgumentDefaultsHelpFormatter,
                                     description='BAO reconstruction on a CUDA device.')
    parser.add_argument('config_fn', action='store', type=str, help='Name of configuration file')
    parser.add_argument('--data-fn', nargs='?', help='Path to input data file (overrides configuration file)')
    parser.add_argument('--randoms-fn', nargs='?', help='Path to input randoms file (overrides configuration file)')
    parser.add_argument('--output-data-fn', nargs='?', help='Path to output data file (overrides configuration file)')
    parser.add_argument('--output-randoms-fn', nargs='?', help='Path to output randoms file (overrides configuration)')
    parser.add_argument('--growth-rate', nargs='?', type=float, help='Logarithmic growth rate (overrides configuration)')
    parser.add_argument('--galaxy-bias', nargs='?', type=float, help='Linear galaxy bias (overrides configuration)')
    opt = parser.parse_args(args=args)
    utils.setup_logging()
    config = load_config(opt.config_fn, **input_config)
    for key, section, value in [('data_fn', 'input', opt.data_fn), ('randoms_fn', 'input', opt.randoms_fn),
                                ('data_fn', 'output', opt.output_data_fn),
                                ('randoms_fn', 'output', opt.output_randoms_fn),
                                ('f', 'cosmology', opt.growth_rate), ('bias', 'cosmology', opt.galaxy_bias)]:
        if value:
            config[section][key] = value
    run(config)
    return 0


if __name__ == '__main__':
    sys.exit(main())
