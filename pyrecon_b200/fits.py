"""
FITS binary tables without fitsio or astropy: what the standalone entry point needs to read and write
catalogues (the reference reads and writes them with fitsio, bin/pyrecon:70-423).

Files follow the FITS standard (version 4.0): 2880-byte blocks of 80-character header cards, an empty
primary HDU, then BINTABLE extensions whose rows are big-endian fields.  Column types: L (bool), B
(uint8), I / J / K (int16 / 32 / 64; with the TZERO offsets of the standard for unsigned integers),
E / D (float32 / 64) and A (strings), each with a repeat count (vector columns such as 3D positions).
"""
import numpy as np

BLOCK = 2880
CARD = 80

# TFORM letter -> big-endian numpy type
_TYPES = {'L': '?', 'B': 'u1', 'I': '>i2', 'J': '>i4', 'K': '>i8', 'E': '>f4', 'D': '>f8'}
# unsigned integers are stored signed with TZERO = 2^(bits - 1)
_UNSIGNED = {'I': ('u2', 1 << 15), 'J': ('u4', 1 << 31), 'K': ('u8', 1 << 63)}


class FITSError(Exception):
    """A file or a column that this reader / writer does not handle."""


def _card(key, value=None, comment=None):
    if value is None:
        text = '{:<8}'.format(key)
    else:
        if isinstance(value, bool):
            v = '{:>20}'.format('T' if value else 'F')
        elif isinstance(value, (int, np.integer)):
            v = '{:>20d}'.format(int(value))
        elif isinstance(value, float):
            v = '{:>20}'.format(repr(value).upper())
        else:
            v = "'{:<8}'".format(str(value).replace("'", "''"))
        text = '{:<8}= {}'.format(key, v)
        if comment:
            text += ' / ' + comment
    if len(text) > CARD:
        raise FITSError('header card too long: {}'.format(text))
    return text.ljust(CARD)


def _header_bytes(cards):
    text = ''.join(cards) + _card('END')
    text += ' ' * (-len(text) % BLOCK)
    return text.encode('ascii')


def _tform(dtype, shape):
    """TFORM and the stored (big-endian) dtype of a column of numpy dtype `dtype` and per-row `shape`."""
    repeat = int(np.prod(shape)) if shape else 1
    kind, size = dtype.kind, dtype.itemsize
    if kind == 'b':
        return '{}L'.format(repeat), np.dtype('?'), None
    if kind == 'f':
        letter = {4: 'E', 8: 'D'}.get(size)
        if letter:
            return '{}{}'.format(repeat, letter), np.dtype(_TYPES[letter]), None
    if kind == 'i':
        letter = {1: 'I', 2: 'I', 4: 'J', 8: 'K'}[size]
        return '{}{}'.format(repeat, letter), np.dtype(_TYPES[letter]), None
    if kind == 'u':
        if size == 1:
            return '{}B'.format(repeat), np.dtype('u1'), None
        letter = {2: 'I', 4: 'J', 8: 'K'}[size]
        return '{}{}'.format(repeat, letter), np.dtype(_TYPES[letter]), _UNSIGNED[letter][1]
    if kind in 'SU':
        width = size if kind == 'S' else size // 4
        return '{}A'.format(width * repeat), np.dtype('S{}'.format(width)), None
    raise FITSError('column type {} not handled'.format(dtype))


def write(fn, columns):
    """Write a dict of columns (first axis: rows), or a structured array, as one BINTABLE extension."""
    if isinstance(columns, np.ndarray):
        columns = {name: columns[name] for name in columns.dtype.names}
    names = list(columns)
    if not names:
        raise FITSError('no columns')
    nrows = len(columns[names[0]])
    fields, cards, stored = [], [], []
    for i, name in enumerate(names, start=1):
        col = np.asarray(columns[name])
        if len(col) != nrows:
            raise FITSError('column {} has {:d} rows, not {:d}'.format(name, len(col), nrows))
        tform, sdt, tzero = _tform(col.dtype, col.shape[1:])
        shape = col.shape[1:] if col.dtype.kind not in 'SU' else ()
        fields.append((name, sdt, shape))
        cards += [_card('TTYPE{:d}'.format(i), name), _card('TFORM{:d}'.format(i), tform)]
        if tzero is not None:
            cards += [_card('TZERO{:d}'.format(i), tzero), _card('TSCAL{:d}'.format(i), 1)]
        if len(shape) > 1:
            cards.append(_card('TDIM{:d}'.format(i), '({})'.format(','.join(str(s) for s in shape[::-1]))))
        if tzero is not None:
            # stored = value - 2^(b - 1), i.e. the value's bits with the sign bit flipped, read as signed
            size = col.dtype.itemsize
            col = (col.astype('u{:d}'.format(size)) ^ np.array(tzero, dtype='u{:d}'.format(size))).view(
                'i{:d}'.format(size))
        elif col.dtype.kind == 'U':
            col = np.char.encode(col, 'ascii')
        stored.append(col)
    table = np.empty(nrows, dtype=[(n, t, s) for n, t, s in fields])
    for (name, _, _), col in zip(fields, stored):
        table[name] = col
    primary = [_card('SIMPLE', True, 'conforms to FITS standard'), _card('BITPIX', 8), _card('NAXIS', 0),
               _card('EXTEND', True)]
    ext = [_card('XTENSION', 'BINTABLE', 'binary table extension'), _card('BITPIX', 8), _card('NAXIS', 2),
           _card('NAXIS1', table.dtype.itemsize), _card('NAXIS2', nrows), _card('PCOUNT', 0), _card('GCOUNT', 1),
           _card('TFIELDS', len(names))] + cards
    data = table.tobytes()
    with open(fn, 'wb') as fh:
        fh.write(_header_bytes(primary))
        fh.write(_header_bytes(ext))
        fh.write(data)
        fh.write(b'\0' * (-len(data) % BLOCK))


def _parse_header(fh):
    """Cards of the next header as {key: value}, or None at the end of the file."""
    out, end = {}, False
    while not end:
        block = fh.read(BLOCK)
        if not block:
            return None
        if len(block) < BLOCK:
            raise FITSError('truncated header')
        text = block.decode('ascii', errors='replace')
        for i in range(0, BLOCK, CARD):
            card = text[i:i + CARD]
            key = card[:8].strip()
            if key == 'END':
                end = True
                break
            if card[8:10] != '= ':
                continue
            value = card[10:]
            if value.lstrip().startswith("'"):
                v = value.lstrip()[1:]
                s, j = '', 0
                while j < len(v):
                    if v[j] == "'":
                        if j + 1 < len(v) and v[j + 1] == "'":
                            s += "'"
                            j += 2
                            continue
                        break
                    s += v[j]
                    j += 1
                out[key] = s.rstrip()
            else:
                v = value.split('/')[0].strip()
                if v in ('T', 'F'):
                    out[key] = v == 'T'
                else:
                    try:
                        out[key] = int(v)
                    except ValueError:
                        out[key] = float(v.replace('D', 'E')) if v else None
    return out


def _data_bytes(h):
    naxis = h.get('NAXIS', 0)
    size = abs(h.get('BITPIX', 8)) // 8
    for a in range(1, naxis + 1):
        size *= h['NAXIS{:d}'.format(a)]
    if naxis == 0:
        size = 0
    size = (size + h.get('PCOUNT', 0)) * h.get('GCOUNT', 1)
    return size + (-size % BLOCK)


def read(fn, columns=None, ext=None):
    """Columns of the first BINTABLE extension (or extension number `ext`) as a dict of numpy arrays in
    native byte order; `columns`: the names to read (all by default)."""
    with open(fn, 'rb') as fh:
        index = 0
        while True:
            h = _parse_header(fh)
            if h is None:
                raise FITSError('{} holds no binary table'.format(fn))
            if h.get('XTENSION') == 'BINTABLE' and (ext is None or ext == index):
                break
            fh.seek(_data_bytes(h), 1)
            index += 1
        nrows, rowbytes, nfields = h['NAXIS2'], h['NAXIS1'], h['TFIELDS']
        raw = np.frombuffer(fh.read(nrows * rowbytes), dtype=np.uint8)
    fields, offset, info = [], 0, {}
    for i in range(1, nfields + 1):
        name, tform = h['TTYPE{:d}'.format(i)], h['TFORM{:d}'.format(i)].strip()
        j = 0
        while j < len(tform) and tform[j].isdigit():
            j += 1
        repeat = int(tform[:j]) if j else 1
        letter = tform[j:j + 1]
        if letter == 'A':
            dt, shape = np.dtype('S{:d}'.format(repeat)), ()
        elif letter in _TYPES:
            dt = np.dtype(_TYPES[letter])
            shape = () if repeat == 1 else (repeat,)
            tdim = h.get('TDIM{:d}'.format(i))
            if tdim:
                shape = tuple(int(s) for s in tdim.strip('()').split(','))[::-1]
        else:
            raise FITSError('TFORM {} of column {} not handled'.format(tform, name))
        fields.append((name, dt, shape))
        info[name] = (letter, h.get('TZERO{:d}'.format(i)), h.get('TSCAL{:d}'.format(i), 1))
        offset += dt.itemsize * (int(np.prod(shape)) if shape else 1)
    if offset != rowbytes:
        raise FITSError('row of {:d} bytes, fields of {:d}'.format(rowbytes, offset))
    table = raw.view(np.dtype([(n, t, s) for n, t, s in fields]))
    out = {}
    for name in (columns if columns is not None else [f[0] for f in fields]):
        if name not in info:
            raise FITSError('no column {} in {}'.format(name, fn))
        letter, tzero, tscal = info[name]
        col = table[name]
        if letter in _UNSIGNED and tzero == _UNSIGNED[letter][1] and tscal == 1:
            size = col.dtype.itemsize
            native = col.astype('i{:d}'.format(size))
            col = native.view('u{:d}'.format(size)) ^ np.array(tzero, dtype='u{:d}'.format(size))
        elif tzero is not None or tscal != 1:
            col = col.astype('f8') * tscal + (tzero or 0)
        elif letter == 'A':
            col = col.copy()
        else:
            col = col.astype(col.dtype.newbyteorder('='))
        out[name] = col
    return out
