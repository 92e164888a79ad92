"""Model serialisation in oneDAL's binary archive format (kmb_model_serialize /
kmb_model_deserialize, host memory: no GPU needed).

Pinned against archives written by oneDAL's own serialisation code
(tests/golden/model_archives.npz, made by the integration client compiled from the
reference sources) and, where that client is built, against it live in both
directions. Malformed archives must fail the way oneDAL's binary_input_archive
does: invalid_argument "Archive content does not match requested type"
(cpp/oneapi/dal/detail/archives.hpp:82-115, detail/array_impl.cpp:39-53)."""
import os
import pickle
import struct
import subprocess

import numpy as np
import pytest

from helpers import GOLDEN
from onedal_b200 import kmeans

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLIENT = os.path.join(ROOT, "integration", "_build", "kmeans_client")
needs_client = pytest.mark.skipif(not os.path.exists(CLIENT), reason="integration client not built")


def _z():
    return np.load(os.path.join(GOLDEN, "model_archives.npz"))


@pytest.mark.parametrize("tag", ["f32", "f64", "wide_f64"])
def test_serialize_writes_onedal_bytes(tag):
    z = _z()
    assert kmeans.model(z[f"C_{tag}"]).serialize() == z[f"archive_{tag}"].tobytes()


def test_serialize_model_without_centroids():
    assert kmeans.model().serialize() == _z()["archive_empty"].tobytes()


@pytest.mark.parametrize("tag", ["f32", "f64", "wide_f64"])
def test_deserialize_reads_onedal_bytes(tag):
    z = _z()
    m = kmeans.model.deserialize(z[f"archive_{tag}"].tobytes())
    C = m.get_centroids()
    assert C.dtype == z[f"C_{tag}"].dtype
    assert np.array_equal(C, z[f"C_{tag}"])
    assert m.get_cluster_count() == z[f"C_{tag}"].shape[0]


def test_deserialize_model_without_centroids():
    m = kmeans.model.deserialize(_z()["archive_empty"].tobytes())
    assert m.get_cluster_count() == 0 and not m.has_centroids()


def test_round_trip_and_pickle():
    rng = np.random.default_rng(7)
    for dt in (np.float32, np.float64):
        for k, d in ((1, 1), (3, 17), (64, 130)):
            C = rng.standard_normal((k, d)).astype(dt)
            m = kmeans.model.deserialize(kmeans.model(C).serialize())
            assert m.get_centroids().dtype == dt and np.array_equal(m.get_centroids(), C)
            p = pickle.loads(pickle.dumps(kmeans.model(C)))
            assert np.array_equal(p.get_centroids(), C)


def _offsets(d):
    """Byte offsets inside a homogen-table model archive with d columns."""
    o = {"magic": 0, "model_nonnull": 4, "model_id": 5, "table_nonnull": 13, "table_id": 14, "meta_nonnull": 22,
         "meta_id": 23, "dtypes_array_id": 31, "dtypes_elem": 39, "dtypes_bytes": 43, "dtypes": 51}
    o["ftypes_array_id"] = o["dtypes"] + 4 * d
    o["ftypes_elem"] = o["ftypes_array_id"] + 8
    o["ftypes_bytes"] = o["ftypes_elem"] + 4
    o["data_array_id"] = o["ftypes_bytes"] + 8 + 4 * d
    o["data_elem"] = o["data_array_id"] + 8
    o["data_bytes"] = o["data_elem"] + 4
    return o


def _patch(b, off, fmt, value):
    b = bytearray(b)
    struct.pack_into(fmt, b, off, value)
    return bytes(b)


@pytest.mark.parametrize("field,fmt,value", [
    ("magic", "<I", 0x4441414E),
    ("model_nonnull", "<B", 0),
    ("model_id", "<Q", 7010000000),        # a linear regression model
    ("table_id", "<Q", 2040000000),        # a CSR table
    ("meta_id", "<Q", 2000000000),         # empty metadata under a homogen table
    ("dtypes_array_id", "<Q", 1),
    ("dtypes_elem", "<i", 0x0008),         # int64 elements where int32 are stored
    ("dtypes_bytes", "<q", 13),            # not a multiple of the element size
    ("ftypes_elem", "<i", 0x0010),
    ("data_elem", "<i", 0x0100),           # float32 elements where uint8 bytes are stored
    ("data_bytes", "<q", 1 << 40),         # past the end
])
def test_malformed_archive_is_invalid_argument(field, fmt, value):
    z = _z()
    good = z["archive_f32"].tobytes()
    bad = _patch(good, _offsets(4)[field], fmt, value)
    with pytest.raises(kmeans.invalid_argument, match="Archive content does not match requested type"):
        kmeans.model.deserialize(bad)


def test_truncated_archive_is_invalid_argument_at_every_length():
    good = _z()["archive_f64"].tobytes()
    for n in range(len(good)):
        with pytest.raises(kmeans.invalid_argument):
            kmeans.model.deserialize(good[:n])


def test_shape_or_type_mismatch_is_invalid_argument():
    good = _z()["archive_f32"].tobytes()
    tail = len(good) - 20                                   # row_count, column_count, layout
    for off, fmt, v in ((tail, "<q", 3), (tail + 8, "<q", 5), (tail + 16, "<i", 0), (tail + 16, "<i", 3)):
        with pytest.raises(kmeans.invalid_argument):
            kmeans.model.deserialize(_patch(good, off, fmt, v))
    mixed = _patch(good, _offsets(4)["dtypes"] + 4, "<i", 0x0200)  # one float64 column among float32
    with pytest.raises(kmeans.invalid_argument):
        kmeans.model.deserialize(mixed)


def test_column_major_table_is_read_row_major():
    """oneDAL homogen tables may be column-major (data_layout::column_major = 2)."""
    C = np.arange(12, dtype=np.float64).reshape(3, 4) * 0.5
    b = bytearray(kmeans.model(C).serialize())
    o = _offsets(4)
    start = o["data_bytes"] + 8
    b[start:start + C.nbytes] = np.ascontiguousarray(C.T).tobytes()
    struct.pack_into("<i", b, len(b) - 4, 2)
    assert np.array_equal(kmeans.model.deserialize(bytes(b)).get_centroids(), C)


@needs_client
@pytest.mark.parametrize("dt,name", [(np.float32, "float"), (np.float64, "double")])
def test_onedal_reads_our_archive_and_we_read_its(tmp_path, dt, name):
    rng = np.random.default_rng(11)
    for k, d in ((1, 1), (5, 3), (40, 129)):
        C = rng.standard_normal((k, d)).astype(dt)
        p = tmp_path / f"ours_{k}.bin"
        p.write_bytes(kmeans.model(C).serialize())
        r = subprocess.run([CLIENT, "deserialize", str(p), name], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0, r.stdout + r.stderr
        lines = dict(l.split(" ", 1) if " " in l else (l, "") for l in r.stdout.splitlines())
        assert int(lines["cluster_count"]) == k
        assert np.array_equal(np.array(lines["centroids"].split(), np.float64).astype(dt), C.ravel())
        src = tmp_path / f"c_{k}.txt"
        src.write_text(f"{k} {d}\n" + " ".join(repr(float(v)) for v in C.ravel()) + "\n")
        out = tmp_path / f"theirs_{k}.bin"
        r = subprocess.run([CLIENT, "serialize", str(src), name, str(out)], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0, r.stdout
        assert out.read_bytes() == kmeans.model(C).serialize()
        assert np.array_equal(kmeans.model.deserialize(out.read_bytes()).get_centroids(), C)


@needs_client
def test_onedal_rejects_what_we_reject(tmp_path):
    """The same malformed archive fails in oneDAL's reader with the same message."""
    good = _z()["archive_f32"].tobytes()
    p = tmp_path / "bad.bin"
    p.write_bytes(_patch(good, _offsets(4)["data_elem"], "<i", 0x0100))
    r = subprocess.run([CLIENT, "deserialize", str(p), "float"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert "Archive content does not match requested type" in r.stdout
