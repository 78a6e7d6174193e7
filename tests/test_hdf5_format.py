"""The HDF5 subset written and read by pyqcm_b200.hdf5 (no HDF5 library in this
environment): round trips of the instance layout's building blocks and checks of
the on-disk structures against the file-format specification."""
import struct

import numpy as np
import pytest


def _tree(H, n_states=40):
    root = H.Group()
    g = root.create_group("cluster_0")
    g.attrs.update({"GS_energy": -12.25, "GS_sectors": "R0:N8:S0:1", "GF_format": "bl", "mixing": 0,
                    "complex_HS": 0, "nstates": n_states})
    p = g.create_group("params")
    p.attrs.update({"U": 4.0, "mu": 2.0, "t": -1.0})
    rng = np.random.default_rng(0)
    for i in range(n_states):
        s = g.create_group(f"state_{i}")
        s.attrs.update({"sec": "R0:N8:S0", "energy": -1.0 * i, "weight": 1.0 / n_states, "gf_format": "bl"})
        b = s.create_group("gf").create_group("block_0")
        b.attrs.update({"L": 3, "M": i})
        b.create_dataset("e", rng.standard_normal(i))
        v = b.create_group("v")
        v.attrs.update({"r": 3, "c": i})
        v.create_dataset("data", rng.standard_normal(3 * i))
    return root


def _same(a, b):
    from pyqcm_b200 import hdf5 as H
    assert type(a) is type(b)
    assert a.attrs.keys() == b.attrs.keys()
    for k in a.attrs:
        assert a.attrs[k] == b.attrs[k] and type(a.attrs[k]) is type(b.attrs[k]), k
    if isinstance(a, H.Dataset):
        assert np.array_equal(a.data, b.data)
        return
    assert sorted(a.keys()) == sorted(b.keys())
    for k in a.keys():
        _same(a.children[k], b.children[k])


def test_round_trip_of_the_instance_layout(tmp_path):
    from pyqcm_b200 import hdf5 as H
    root = _tree(H)
    path = str(tmp_path / "inst.h5")
    H.write_file(path, root)
    _same(root, H.read_file(path))
    # 'a' mode keeps what is there and replaces a group
    with H.File(path, "a") as f:
        f.root.unlink("cluster_0")
        f.root.create_group("cluster_0").attrs["nstates"] = 0
        f.root.create_group("cluster_1").create_dataset("x", [1.0, 2.0])
    r = H.read_file(path)
    assert r.group("cluster_0").attrs == {"nstates": 0} and list(r.group("cluster_1").dataset("x")) == [1.0, 2.0]


def test_on_disk_structures_follow_the_specification(tmp_path):
    """Superblock version 0 with 8-byte offsets and lengths and the root group's
    symbol-table entry; groups as symbol tables (a TREE node of SNOD children,
    names sorted and stored in a HEAP whose free list is empty); attribute,
    dataspace, datatype and layout messages with the version-1/-3 encodings."""
    from pyqcm_b200 import hdf5 as H
    path = str(tmp_path / "s.h5")
    H.write_file(path, _tree(H, 20))
    d = open(path, "rb").read()
    assert d[:8] == b"\x89HDF\r\n\x1a\n" and d[8] == 0 and d[13] == 8 and d[14] == 8
    leaf_k, internal_k = struct.unpack_from("<HH", d, 16)
    assert struct.unpack_from("<Q", d, 40)[0] == len(d)  # end-of-file address
    root_oh, cache = struct.unpack_from("<QI", d, 64)
    btree, heap = struct.unpack_from("<QQ", d, 80)
    assert cache == 1 and d[btree:btree + 4] == b"TREE" and d[heap:heap + 4] == b"HEAP"
    assert struct.unpack_from("<Q", d, heap + 16)[0] == 1  # empty free list
    assert d[root_oh] == 1  # version 1 object header
    nmsg = struct.unpack_from("<H", d, root_oh + 2)[0]
    assert struct.unpack_from("<HH", d, root_oh + 16) == (0x0011, 16)  # symbol table message first
    # the cluster group: 21 links (params + 20 states) over two symbol-table nodes, names in byte order
    r = H._Reader(d)
    links = r.links(btree, heap)
    assert [n for n, _ in links] == ["cluster_0"]
    msgs = r.messages(links[0][1])
    bt, lh = struct.unpack_from("<QQ", [b for t, b, _ in msgs if t == 0x0011][0], 0)
    names = [n for n, _ in r.links(bt, lh)]
    assert names == sorted(names) and len(names) == 21 and names[:3] == ["params", "state_0", "state_1"]
    assert struct.unpack_from("<H", d, bt + 6)[0] == 2 and leaf_k == 8 and internal_k == 64
    # attributes: a double, an int and a fixed-length string
    attrs = dict(r.attribute(b) for t, b, _ in msgs if t == 0x000C)
    assert attrs["GS_energy"] == -12.25 and attrs["nstates"] == 20 and attrs["GS_sectors"] == "R0:N8:S0:1"


def test_refuses_what_it_does_not_read(tmp_path):
    from pyqcm_b200 import hdf5 as H
    p = tmp_path / "bad.h5"
    p.write_bytes(b"not an hdf5 file at all" + b"\0" * 100)
    with pytest.raises(ValueError):
        H.read_file(str(p))
    g = H.Group()
    g.create_group("a")
    with pytest.raises(ValueError):
        g.create_dataset("a", [1.0])
