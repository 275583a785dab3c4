"""The Streamable ASCII interchange (ves3d_b200/streamable.py) against the reference's own
writer and reader (oracle/_ref/ref_stream, compiled from src/Array.cc, Scalars.cc and
Vectors.cc): the golden text re-packs byte for byte, the reference reads what this writer
produces, the reference's older header forms parse, and surfaces round-trip. CPU only."""
import os
import subprocess

import numpy as np
import pytest

from ves3d_b200 import streamable as st

HERE = os.path.dirname(os.path.abspath(__file__))
REF_STREAM = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_stream")


def golden():
    return open(os.path.join(HERE, "golden", "ref_stream_p4.txt")).read()


def test_golden_vectors_and_scalars_repack_byte_for_byte():
    text = golden()
    tok = st.Tokens(text)
    v = st.unpack_vectors(tok)
    s = st.unpack_scalars(tok)
    assert (v["name"], v["p"], v["n_vec"], v["order"], v["stride"]) == ("position", 4, 2, "AxisMajor", 40)
    assert v["data"].size == 2 * 3 * 40 and s["data"].size == 2 * 40 and s["name"] == "tension"
    # the reference's values: sin(0.37 i) + 1e-3 i and cos(0.11 i) / (1 + i)
    i = np.arange(v["data"].size)
    assert np.abs(v["data"] - (np.sin(0.37 * i) + 1e-3 * i)).max() < 1e-15
    ours = st.pack_vectors(v["name"], v["data"], 4, 2, v["order"]) + st.pack_scalars(s["name"], s["data"], 4, 2)
    assert ours == text


@pytest.mark.skipif(not os.path.exists(REF_STREAM), reason="oracle/_ref/ref_stream not built")
def test_reference_reads_what_this_writer_produces(tmp_path):
    rng = np.random.default_rng(7)
    p, n = 6, 3
    X = rng.standard_normal(n * 3 * 2 * p * (p + 1)) * 10.0 ** rng.integers(-8, 8, size=n * 3 * 2 * p * (p + 1))
    text = st.pack_vectors("position", X, p, n)
    src, dst = tmp_path / "in.txt", tmp_path / "out.txt"
    src.write_text(text)
    subprocess.check_call([REF_STREAM, "vectors", str(src), str(dst)], env=dict(os.environ, VES3D_DIR="/"))
    assert dst.read_text() == text
    back = st.unpack_vectors(st.Tokens(dst.read_text()))
    assert np.array_equal(back["data"], X)  # 17 significant digits round-trip FP64 exactly


def test_older_header_forms():
    """A version followed by '+', and the pre-591 layout whose VECTORS and SCALARS headers
    carry a name (src/Vectors.cc:104-117, src/Scalars.cc:242-256)."""
    data = np.arange(2 * 3 * 12, dtype=float) / 7
    text = st.pack_vectors("x", data, 2, 2, version=812)
    plus = text.replace("version: 812", "version: 812 +")
    assert np.array_equal(st.unpack_vectors(st.Tokens(plus))["data"], data)
    old = text.replace("VECTORS\nversion: 812\n", "VECTORS\nversion: 500\nname: x\n").replace(
        "SCALARS\nversion: 812\n", "SCALARS\nversion: 500\nname: x\n").replace("ARRAY\nversion: 812", "ARRAY\nversion: 500")
    v = st.unpack_vectors(st.Tokens(old))
    assert np.array_equal(v["data"], data) and v["p"] == 2
    with pytest.raises(ValueError):
        st.unpack_vectors(st.Tokens(text.replace("/ARRAY", "/ARR")))


def test_surface_blocks_round_trip_and_point_major():
    from ves3d_b200 import workloads
    X, _ = workloads.suspension(2, 6, 3.0, seed=3)
    p, n = 6, X.size // (3 * 84)
    text = "PARAMETERS ... /PARAMETERS\n" + st.pack_surface("surface", X, p, n) + "EVOLVE ... \n"
    surfs = st.read_surfaces(text)
    assert len(surfs) == 1 and surfs[0]["p"] == p and surfs[0]["n_vec"] == n
    assert surfs[0]["settings"]["diff_filter_freq"] == "4" and surfs[0]["settings"]["SHT_resample_order"] == "12"
    assert np.array_equal(surfs[0]["X"], X)
    # point-major data comes back AxisMajor
    pm = X.reshape(n, 3, 84).transpose(0, 2, 1).reshape(-1)
    text_pm = st.pack_surface("surface", X, p, n).replace(st.pack_vectors("position", X, p, n, "AxisMajor"),
                                                         st.pack_vectors("position", pm, p, n, "PointMajor"))
    assert np.array_equal(st.read_surfaces(text_pm)[0]["X"], X)
