"""The built-in FITS binary-table reader / writer (pyrecon_b200.fits): layout of the file against the
FITS standard's rules, and round trips of every column type the catalogues use."""
import numpy as np
import pytest


def test_roundtrip_all_types(tmp_path):
    from pyrecon_b200 import fits
    rng = np.random.default_rng(1)
    n = 1001
    cols = {'Position': rng.uniform(-1e3, 1e3, (n, 3)), 'Weight': rng.uniform(0.5, 1.5, n).astype('f4'),
            'Z': rng.uniform(0., 2., n), 'ID': np.arange(n, dtype='i8') - 500, 'FLAG': rng.integers(0, 2, n).astype(bool),
            'NTILE': rng.integers(0, 200, n).astype('u1'), 'SHORT': rng.integers(-3000, 3000, n).astype('i2'),
            'U16': rng.integers(0, 65535, n).astype('u2'), 'U32': rng.integers(0, 2 ** 32 - 1, n, dtype='u8').astype('u4'),
            'U64': rng.integers(0, 2 ** 63, n, dtype='u8') * np.uint64(2), 'NAME': np.array(['gal{:d}'.format(i) for i in range(n)]),
            'M': rng.standard_normal((n, 2, 3)).astype('f4')}
    fn = str(tmp_path / 'cat.fits')
    fits.write(fn, cols)
    raw = open(fn, 'rb').read()
    assert len(raw) % 2880 == 0
    assert raw[:80].decode() == 'SIMPLE  = {:>20} / conforms to FITS standard'.format('T').ljust(80)
    assert raw[2880:2960].decode().startswith("XTENSION= 'BINTABLE'")
    got = fits.read(fn)
    assert list(got) == list(cols)
    for k, v in cols.items():
        g = got[k]
        if v.dtype.kind == 'U':
            assert g.astype('U').tolist() == v.tolist()
        else:
            assert g.dtype == v.dtype and g.shape == v.shape, (k, g.dtype, g.shape)
            np.testing.assert_array_equal(g, v, err_msg=k)
    sub = fits.read(fn, columns=['Z', 'Position'])
    assert list(sub) == ['Z', 'Position'] and np.array_equal(sub['Position'], cols['Position'])
    with pytest.raises(fits.FITSError):
        fits.read(fn, columns=['NOPE'])


def test_reads_a_handwritten_file(tmp_path):
    """A file laid out by hand from the standard (cards, big-endian rows, block padding, an image HDU
    before the table) reads back as written."""
    from pyrecon_b200 import fits

    def header(cards):
        text = ''.join(c.ljust(80) for c in cards + ['END'])
        return (text + ' ' * (-len(text) % 2880)).encode()
    rows = np.zeros(3, dtype=[('X', '>f8'), ('N', '>i4'), ('T', 'S4')])
    rows['X'] = [1.5, -2.25, 3e10]
    rows['N'] = [7, -8, 2 ** 30]
    rows['T'] = [b'ab', b'cd', b"e'f"]
    image = np.arange(6, dtype='>i2').tobytes()
    blob = header(['SIMPLE  =                    T', 'BITPIX  =                    8', 'NAXIS   =                    0',
                   'EXTEND  =                    T'])
    blob += header(['XTENSION= \'IMAGE   \'', 'BITPIX  =                   16', 'NAXIS   =                    2',
                    'NAXIS1  =                    3', 'NAXIS2  =                    2', 'PCOUNT  =                    0',
                    'GCOUNT  =                    1'])
    blob += image + b'\0' * (-len(image) % 2880)
    blob += header(["XTENSION= 'BINTABLE'", 'BITPIX  =                    8', 'NAXIS   =                    2',
                    'NAXIS1  =                   16', 'NAXIS2  =                    3', 'PCOUNT  =                    0',
                    'GCOUNT  =                    1', 'TFIELDS =                    3', "TTYPE1  = 'X       '",
                    "TFORM1  = '1D      '", "TTYPE2  = 'N       '", "TFORM2  = 'J       ' / a comment",
                    "TTYPE3  = 'T       '", "TFORM3  = '4A      '"])
    blob += rows.tobytes() + b'\0' * (-rows.nbytes % 2880)
    fn = str(tmp_path / 'hand.fits')
    open(fn, 'wb').write(blob)
    got = fits.read(fn)
    np.testing.assert_array_equal(got['X'], [1.5, -2.25, 3e10])
    np.testing.assert_array_equal(got['N'], [7, -8, 2 ** 30])
    assert got['T'].tolist() == [b'ab', b'cd', b"e'f"]
