"""A reader of Tecplot binary flowfield files (the published version-112 layout, ordered zones,
double data, no auxiliary data), written here independently of the library to check the files it
writes and the reference's own."""
import struct

import numpy as np


class _Buf:
    def __init__(self, data):
        self.d, self.o = data, 0

    def take(self, fmt):
        v = struct.unpack_from("<" + fmt, self.d, self.o)
        self.o += struct.calcsize("<" + fmt)
        return v if len(v) > 1 else v[0]

    def string(self):
        out = []
        while True:
            c = self.take("i")
            if c == 0:
                return "".join(out)
            out.append(chr(c))


def read(path):
    """{"title", "names", "zones": [{"name", "time", "dims", "minmax", "data": {name: array[k, j, i]}}]}"""
    with open(path, "rb") as f:
        b = _Buf(f.read())
    magic = b.d[:8]
    assert magic == b"#!TDV112", magic
    b.o = 8
    assert b.take("i") == 1
    file_type = b.take("i")
    title = b.string()
    n_var = b.take("i")
    names = [b.string() for _ in range(n_var)]
    zones = []
    while True:
        marker = b.take("f")
        if marker == 357.0:
            break
        assert marker == 299.0, marker
        z = {"name": b.string()}
        z["parent"], z["strand"] = b.take("ii")
        z["time"] = b.take("d")
        z["color"], z["type"], z["var_loc"], z["raw_faces"], z["misc_faces"] = b.take("iiiii")
        z["dims"] = b.take("iii")
        z["aux"] = b.take("i")
        zones.append(z)
    for z in zones:
        assert b.take("f") == 299.0
        z["formats"] = [b.take("i") for _ in range(n_var)]
        z["passive"], z["sharing"], z["share_conn"] = b.take("iii")
        z["minmax"] = [b.take("dd") for _ in range(n_var)]
        ni, nj, nk = z["dims"]
        n = ni * nj * nk
        z["data"] = {}
        for name in names:
            a = np.frombuffer(b.d, dtype="<f8", count=n, offset=b.o).reshape(nk, nj, ni).copy()
            b.o += 8 * n
            z["data"][name] = a
    assert b.o == len(b.d), (b.o, len(b.d))
    return {"file_type": file_type, "title": title, "names": names, "zones": zones}
