"""Writer for ZDF diagnostic files from Python: grid files
``<path>/<name>-<iter:06>.zdf`` and particle files
``<path>/particles-<name>-<iter:06>.zdf``, with the record layout the
reference's zdf.c writes and its zdf.py reads (zdf.h:20-200): the magic
``ZDF1``, then records {uint32 id, string name, uint64 length, payload};
strings are a uint32 length and the bytes padded to 4; little-endian.  Byte
for byte the same as the library's C++ writer (cpp/zdf.h)."""
import os
import struct

import numpy as np

STRING_ID = 0x00030000
DATASET_ID = 0x00100002
ITERATION_ID = 0x00200001
GRID_INFO_ID = 0x00210001
PART_INFO_ID = 0x00220002
FLOAT32 = 9


def _pad4(n):
    return (n + 3) // 4 * 4


def _str(s):
    b = s.encode()
    return struct.pack('<I', len(b)) + b + b'\0' * (_pad4(len(b)) - len(b))


def _record(rid, name, payload):
    return struct.pack('<I', rid) + _str(name) + struct.pack('<Q', len(payload)) + payload


def _iteration(n, t, time_units, name='ITERATION'):
    return _record(ITERATION_ID, name or 'Iteration', struct.pack('<id', int(n), float(t)) + _str(time_units))


def _dataset(name, data, index):
    data = np.ascontiguousarray(data, np.float32)
    count = tuple(reversed(data.shape))            # x fastest
    head = struct.pack('<IiI', index, FLOAT32, len(count)) + struct.pack('<%dQ' % len(count), *count)
    return _record(DATASET_ID, name, head + data.tobytes())


def grid_info(name, count, label, units, axes):
    """axes: list of (name, min, max, label, units), one per dimension (or empty)."""
    p = struct.pack('<I', len(count)) + struct.pack('<%dQ' % len(count), *count)
    p += _str(label) + _str(units) + struct.pack('<i', 1 if axes else 0)
    for a in axes:
        p += _str(a[0]) + struct.pack('<idd', 0, float(a[1]), float(a[2])) + _str(a[3]) + _str(a[4])
    return _record(GRID_INFO_ID, name, p)


def save_grid(data, name, label, units, axes, n, t, path, time_units='1/\\omega_n', iter_name=''):
    """One float32 grid (numpy array, shape [ny, nx] or [nx]) as <path>/<name>-<n:06>.zdf.
    The iteration record is named iter_name ('Iteration' when empty, as the
    field and current files of the reference; 'ITERATION' for charge and
    phase-space files)."""
    data = np.asarray(data, np.float32)
    os.makedirs(path, exist_ok=True)
    fn = os.path.join(path, '%s-%06d.zdf' % (name, n))
    with open(fn, 'wb') as f:
        f.write(b'ZDF1')
        f.write(_record(STRING_ID, 'TYPE', _str('grid')))
        f.write(grid_info(name, tuple(reversed(data.shape)), label, units, axes))
        f.write(_iteration(n, t, time_units, iter_name))
        f.write(_dataset(name, data, 1))
    return fn


def save_particles(quants, name, label, qnames, qlabels, qunits, n, t, path, time_units='1/\\omega_n'):
    """Particle quantities (list of 1D float32 arrays) as <path>/particles-<name>-<n:06>.zdf."""
    os.makedirs(path, exist_ok=True)
    fn = os.path.join(path, 'particles-%s-%06d.zdf' % (name, n))
    np_ = len(quants[0]) if quants else 0
    info = _str(label) + struct.pack('<QI', np_, len(qnames))
    for group in (qnames, qlabels, qunits):
        for q in group:
            info += _str(q)
    with open(fn, 'wb') as f:
        f.write(b'ZDF1')
        f.write(_record(STRING_ID, 'TYPE', _str('particles')))
        f.write(_record(PART_INFO_ID, name, info))
        f.write(_iteration(n, t, time_units, ''))
        for k, (q, d) in enumerate(zip(qnames, quants)):
            f.write(_dataset(q, d, k + 1))
    return fn
