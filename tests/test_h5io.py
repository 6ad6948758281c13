"""The HDF5 codec (icempm_3dm_b200.h5io) against the reference's own raw
point cloud (build/geometries_3d/3d_200k.h5, written by the HDF5 library),
and write -> read round trips.

The reference file pins the reader: every chunk is a zlib stream whose
Adler-32 checksum is verified on decompression, the datatype and dataspace
come from the file's messages, and the 'volume' attribute (3.75 m^3) is
independently consistent with the coordinates' bounding box (2.5 x 1 x 1.5).
It also pins the writer: for the same dataset description the writer's
dataspace, datatype, fill value, filter pipeline, layout and attribute
messages equal the library's byte for byte (addresses aside)."""
import os

import numpy as np
import pytest

from icempm_3dm_b200 import h5io

from oracle import pyoracle as po  # noqa: E402

# the tree oracle/_ref was built from, if it is on this machine
REF_H5 = os.path.join(po.reference_tree() or "", "build", "geometries_3d", "3d_200k.h5")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_H5), reason="reference point cloud not present")


@needs_ref
def test_reads_the_reference_point_cloud():
    with h5io.H5File(REF_H5) as f:
        assert f.keys() == ["llGrainIDs", "x", "y", "z"]
        g = f.read("llGrainIDs")
        xyz = [f.read(k) for k in "xyz"]
        vol = f.attrs("llGrainIDs")["volume"]
    n = 202329
    assert g.dtype == np.uint64 and g.shape == (n,)
    assert g.min() == 0 and g.max() == 999 and np.unique(g).size == 1000
    for c, L in zip(xyz, (2.5, 1.0, 1.5)):
        assert c.dtype == np.float64 and c.shape == (n,)
        assert 0.0 <= c.min() < 1e-4 and L - 1e-4 < c.max() <= L
    box = np.prod([c.max() - c.min() for c in xyz])
    assert vol == 3.75
    assert abs(box - vol) / vol < 1e-4


def _messages(f, name):
    return [(t, fl, d) for t, fl, d in f._messages(f._datasets[name]) if t != 0x12]


@needs_ref
def test_writer_encodes_messages_like_the_hdf5_library(tmp_path):
    with h5io.H5File(REF_H5) as ref:
        x = ref.read("x")
        g = ref.read("llGrainIDs")
        lay = h5io._parse_layout([d for t, fl, d in _messages(ref, "x") if t == 0x08][0])
        chunk = lay[2][0]
        level = [d for t, fl, d in _messages(ref, "x") if t == 0x0B][0][24]
        out = tmp_path / "pc.h5"
        with h5io.H5Writer(out) as w:
            w.create_dataset("llGrainIDs", g, chunks=(chunk,), deflate=level, attrs={"volume": np.float64(3.75)})
            w.create_dataset("x", x, chunks=(chunk,), deflate=level)
        with h5io.H5File(out) as mine:
            for name in ("llGrainIDs", "x"):
                a, b = _messages(ref, name), _messages(mine, name)
                assert [(t, fl) for t, fl, _ in a] == [(t, fl) for t, fl, _ in b], name
                for (t, fl, da), (_, _, db) in zip(a, b):
                    if t == 0x08:   # layout: the chunk index address differs
                        assert da[:3] == db[:3] and da[11:] == db[11:]
                    else:
                        assert da == db, (name, hex(t))
            assert np.array_equal(mine.read("x"), x)
            assert np.array_equal(mine.read("llGrainIDs"), g)


@needs_ref
def test_reference_data_survives_a_rewrite_in_every_layout(tmp_path):
    with h5io.H5File(REF_H5) as ref:
        data = {k: ref.read(k) for k in ref.keys()}
    for mode, kw in (("contig", {}), ("chunk", {"chunks": (4096,)}), ("deflate", {"chunks": (50000,), "deflate": 5})):
        p = tmp_path / f"{mode}.h5"
        with h5io.H5Writer(p) as w:
            for k, v in data.items():
                w.create_dataset(k, v, **kw)
        with h5io.H5File(p) as f:
            assert f.keys() == sorted(data)
            for k, v in data.items():
                r = f.read(k)
                assert r.dtype == v.dtype and np.array_equal(r, v), (mode, k)


def test_round_trip_types_ranks_layouts_and_attributes(tmp_path):
    rng = np.random.default_rng(0)
    sets = {
        "f8": rng.standard_normal(1000),
        "f4": rng.standard_normal((30, 7)).astype(np.float32),
        "i4": rng.integers(-2**31, 2**31 - 1, 513, dtype=np.int32),
        "u4": rng.integers(0, 2**32 - 1, 77, dtype=np.uint32),
        "u1": rng.integers(0, 255, 9, dtype=np.uint8),
        "u8": rng.integers(0, 2**63, 100, dtype=np.uint64),
        "i8": rng.integers(-2**62, 2**62, (5, 4, 3), dtype=np.int64),
        "many_chunks": rng.standard_normal(10_000),       # 100 chunks: a two-level chunk index
        "big_chunks": np.arange(200_000, dtype=np.float64),
        "one": np.array([42.0]),
    }
    layouts = {"many_chunks": dict(chunks=(100,), deflate=5), "big_chunks": dict(chunks=(1 << 16,), deflate=1),
               "f4": dict(chunks=(8, 3)), "i8": dict(chunks=(2, 4, 2), deflate=9)}
    attrs = {"a_int": np.int32(-7), "a_uint": np.uint32(4000000000), "a_u8": np.uint8(1), "a_dbl": np.float64(0.1),
             "a_u64": np.uint64(2**63 + 5), "a_vec": np.arange(3, dtype=np.float64)}
    p = tmp_path / "t.h5"
    with h5io.H5Writer(p) as w:
        for k, v in sets.items():
            w.create_dataset(k, v, attrs=attrs if k == "f8" else None, **layouts.get(k, {}))
        for i in range(11):                        # more names than one symbol table node holds
            w.create_dataset(f"extra{i:02d}", np.full(3, i, dtype=np.int32))
    with h5io.H5File(p) as f:
        assert len(f.keys()) == len(sets) + 11
        for k, v in sets.items():
            r = f.read(k)
            assert r.dtype == v.dtype and r.shape == v.shape and np.array_equal(r, v), k
        for i in range(11):
            assert np.array_equal(f.read(f"extra{i:02d}"), np.full(3, i, dtype=np.int32))
        got = f.attrs("f8")
        assert list(got) == list(attrs)
        for k, v in attrs.items():
            assert np.asarray(got[k]).dtype == np.asarray(v).dtype
            assert np.array_equal(got[k], v), k
        assert f.attrs("u1") == {}


def test_reader_rejects_what_it_does_not_read(tmp_path):
    p = tmp_path / "bad.h5"
    p.write_bytes(b"\x89HDF\r\n\x1a\n" + bytes([2]) + b"\0" * 200)
    with pytest.raises(h5io.H5Error, match="superblock version 2"):
        h5io.H5File(p)
    q = tmp_path / "none.h5"
    q.write_bytes(b"\0" * 4096)
    with pytest.raises(h5io.H5Error, match="no HDF5 signature"):
        h5io.H5File(q)
    with pytest.raises(h5io.H5Error):
        with h5io.H5Writer(tmp_path / "c.h5") as w:
            w.create_dataset("s", np.array(["a"]))


@needs_ref
def test_damaged_copies_of_the_reference_file_raise_and_do_not_hang(tmp_path):
    """Truncations and byte corruptions of a real file end in an exception
    (H5Error, or an index/value error from numpy on garbage), never in a hang."""
    data = bytearray(open(REF_H5, "rb").read())
    rng = np.random.default_rng(0)
    cases = [data[:n] for n in (100, 700, 1100, 5000, 300000, len(data) // 2)]
    for _ in range(40):
        d = bytearray(data)
        for pos in rng.integers(0, 3000, 4):        # metadata region: superblock, heap, B-trees, headers
            d[pos] = rng.integers(0, 256)
        cases.append(d)
    for k, d in enumerate(cases):
        p = tmp_path / f"d{k}.h5"
        p.write_bytes(bytes(d))
        try:
            with h5io.H5File(p) as f:
                for name in f.keys():
                    f.read(name)
                    f.attrs(name)
        except (h5io.H5Error, KeyError, ValueError, IndexError, UnicodeDecodeError, OverflowError, TypeError,
                MemoryError):
            pass


def test_writer_rejects_names_outside_the_root_group(tmp_path):
    with pytest.raises(h5io.H5Error):
        with h5io.H5Writer(tmp_path / "n.h5") as w:
            w.create_dataset("a/b", np.zeros(3))


def test_deflated_chunks_do_not_depend_on_the_thread_count(tmp_path, monkeypatch):
    """Chunks are compressed and decoded on a pool of threads: the file's bytes
    are those of a one-thread write, and the data reads back exactly."""
    rng = np.random.default_rng(7)
    data = rng.standard_normal((37, 5000)).astype(np.float32)
    data[:, ::3] = 0.0                                   # something for deflate to find

    def write(path):
        with h5io.H5Writer(path) as w:
            w.create_dataset("A", data, chunks=(8, 1024), deflate=5)
            w.create_dataset("B", data.reshape(-1)[:70001], chunks=(4096,), deflate=1)
        return path.read_bytes()

    many = write(tmp_path / "many.h5")
    monkeypatch.setattr(os, "cpu_count", lambda: 1)
    one = write(tmp_path / "one.h5")
    assert many == one
    monkeypatch.undo()
    with h5io.H5File(tmp_path / "many.h5") as f:
        assert np.array_equal(f.read("A"), data)
        assert np.array_equal(f.read("B"), data.reshape(-1)[:70001])
