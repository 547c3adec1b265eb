"""The .qttb layout (TravelTimeTable.Write/Open) and the header document, on the CPU."""
import hashlib

import numpy as np

from oracle import qttb as OQ
from tomostar_b200 import qttb
from tomostar_b200 import synthetic as syn
from tomostar_b200.grid import GridDef


def test_layout_known_answers():
    # 12 bytes of magic and length, the JSON, then zeros to the next multiple of 64 (:65, :108).
    assert [qttb.data_offset(n) for n in (0, 52, 53, 116, 117)] == [64, 64, 128, 128, 192]
    data = OQ.write_bytes(b"{}", [1.5, np.nan, -np.inf, np.inf, 1e300, 2.0])
    assert data[:8] == b"QTTB\x01\x00\x00\x00" and data[8:12] == b"\x02\x00\x00\x00" and len(data) == 64 + 24
    h, v = OQ.open_bytes(data)
    assert h == b"{}" and list(v[[0, 5]]) == [1.5, 2.0]
    assert np.isposinf(v[1:4]).all() and np.isposinf(v[4])  # 1e300 overflows float to +inf


def test_header_document():
    """TomoJson.Options (Model/Basics.cs:60-75): indented, properties in declaration order, the enum by
    name, numbers in .NET's shortest round-trip layout."""
    g = GridDef(13.0, 13.5, 42.25, 43.0, -2.0, 20.0, 21, 31, 12)
    want = ('{\n  "StationId": "IV.NRCA",\n  "Phase": "S",\n  "Lon": 13.1234,\n  "Lat": 42.5,\n  "DepthKm": -1.25,\n'
            '  "Grid": {\n    "MinLon": 13,\n    "MaxLon": 13.5,\n    "MinLat": 42.25,\n    "MaxLat": 43,\n'
            '    "MinDepthKm": -2,\n    "MaxDepthKm": 20,\n    "Nx": 21,\n    "Ny": 31,\n    "Nz": 12\n  },\n'
            '  "ModelKey": "ABC",\n  "Solver": "fast sweeping \\u002B cuda"\n}')
    got = qttb.header_json("IV.NRCA", "S", 13.1234, 42.5, -1.25, g, "ABC", "fast sweeping + cuda")
    assert got.decode() == want
    assert [qttb.net_number(x) for x in (1e-5, 1e15, 123456789012345.0, -0.0, 0.1, 1.5e-7)] == \
        ["1E-05", "1E+15", "123456789012345", "-0", "0.1", "1.5E-07"]


def test_model_key_composition():
    """ForwardModel.Key (:176-183): SHA-256 of the slowness bytes then the grid's JSON, 32 upper-case hex."""
    job = syn.relocation_small()
    s = job.slowness[0]
    k = qttb.model_key(job.grid, s)
    assert len(k) == 32 and k == k.upper()
    assert k == hashlib.sha256(s.astype("<f8").tobytes() + qttb.grid_json(job.grid)).hexdigest().upper()[:32]
    assert k != qttb.model_key(job.grid, job.slowness[1])


def test_header_escapes_and_numbers():
    """The default encoder's escapes (HTML-sensitive and non-ASCII characters as \\uXXXX, control
    characters short) and .NET's number layout for negatives and exponents."""
    g = GridDef(-1.0, 1.0, -1.0, 1.0, 0.0, 5.0, 3, 3, 3)
    h = qttb.header_json('A"B<é>\n', "P", -0.000012, -1e16, 0.5, g).decode()
    assert '"StationId": "A\\u0022B\\u003C\\u00E9\\u003E\\n"' in h
    assert '"Lon": -1.2E-05' in h and '"Lat": -1E+16' in h and '"DepthKm": 0.5' in h
    assert '"MinLon": -1' in h and '"Nz": 3\n  }' in h
