"""Minimal ZDF reader for the tests (records: uint32 id, string name, uint64
length, payload; strings padded to 4 bytes; little-endian)."""
import struct

import numpy as np


def _str(b, o):
    n = struct.unpack_from('<I', b, o)[0]
    o += 4
    s = b[o:o + n].decode()
    return s, o + ((n + 3) // 4) * 4


def read(path):
    b = open(path, 'rb').read()
    assert b[:4] == b'ZDF1'
    o = 4
    out = {'datasets': {}}
    while o < len(b):
        rid = struct.unpack_from('<I', b, o)[0]
        name, o = _str(b, o + 4)
        length = struct.unpack_from('<Q', b, o)[0]
        o += 8
        p = o
        if rid == 0x00030000:
            out[name] = _str(b, p)[0]
        elif rid == 0x00200001:
            n, t = struct.unpack_from('<id', b, p)
            out['iteration'] = {'name': name, 'n': n, 't': t}
        elif rid == 0x00210001:
            nd = struct.unpack_from('<I', b, p)[0]
            cnt = struct.unpack_from('<%dQ' % nd, b, p + 4)
            label, q = _str(b, p + 4 + 8 * nd)
            units, q = _str(b, q)
            has_axis = struct.unpack_from('<i', b, q)[0]
            q += 4
            axes = []
            for _ in range(nd if has_axis else 0):
                aname, q = _str(b, q)
                atype, amin, amax = struct.unpack_from('<idd', b, q)
                alabel, q = _str(b, q + 20)
                aunits, q = _str(b, q)
                axes.append({'name': aname, 'type': atype, 'min': amin, 'max': amax,
                             'label': alabel, 'units': aunits})
            out['grid'] = {'name': name, 'ndims': nd, 'count': cnt, 'label': label, 'units': units,
                           'axis': axes}
        elif rid == 0x00220002:
            label, q = _str(b, p)
            np_ = struct.unpack_from('<Q', b, q)[0]
            out['particles'] = {'name': name, 'label': label, 'np': np_}
        elif rid == 0x00100002:
            _, dtype, nd = struct.unpack_from('<IiI', b, p)
            cnt = struct.unpack_from('<%dQ' % nd, b, p + 12)
            q = p + 12 + 8 * nd
            n = int(np.prod(cnt))
            data = np.frombuffer(b, np.float32, n, q)
            out['datasets'][name] = data.reshape(tuple(reversed(cnt)))
        o = p + length
    return out
