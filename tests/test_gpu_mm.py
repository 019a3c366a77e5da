"""Matrix Market into a device CSR handle and back (sk_matrix_market_read,
sk_matrix_market_read_buffer, sk_matrix_market_write), held bit for bit
against the reference's read_matrix_market + to_compressed_row and
write_matrix_market (golden fixtures and the reference's Catch2 cases), and
at full size through a lossless round trip."""
import numpy as np
import pytest

from sparkit_b200 import _lib, gpu, matgen
from tests.golden.make_golden import mm_texts
from tests.helpers import csr_from_entries

pytestmark = pytest.mark.gpu


def _same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_read_write_match_reference_fixtures(gpu_lib, golden, dtype, tmp_path):
    """Every fixture text from a buffer and from a file, with 1 and 7
    parsing threads: the same CSR arrays as the reference, the sign of zero
    included; writing the result gives the reference's bytes."""
    dt = np.dtype(dtype)
    for name in mm_texts():
        text = bytes(golden[f"mm/{name}/text"])
        tag = f"mm/{name}/{dtype}"
        path = tmp_path / f"{name}.mtx"
        path.write_bytes(text)
        for src, threads in ((text, 1), (text, 7), (path, 0)):
            Ad = gpu.read_matrix_market(src, dt, threads)
            A = Ad.to_host()
            assert A.shape() == tuple(golden[f"{tag}/shape"]), name
            for f in ("row_ptr", "col_ind", "values"):
                assert _same_bits(getattr(A, f)(), golden[f"{tag}/{f}"]), (name, threads, f)
        out = tmp_path / f"{name}.out.mtx"
        gpu.write_matrix_market(Ad, out)
        assert out.read_bytes() == bytes(golden[f"{tag}/written"]), name


def test_known_answers(gpu_lib, known, tmp_path):
    """The reference's own test cases (matrix_market_test.cpp)."""
    mm = known["matrix_market"]
    for case in mm["read"]:
        A = gpu.read_matrix_market(case["text"].encode()).to_host()
        D = np.zeros(case["shape"])
        for r, c, v in case["entries"]:
            D[r, c] = v
        rp, ci, va = A.row_ptr(), A.col_ind(), A.values()
        G = np.zeros(case["shape"])
        for r in range(A.shape()[0]):
            G[r, ci[rp[r]:rp[r + 1]]] = va[rp[r]:rp[r + 1]]
        assert np.array_equal(G, D), case["source"]
    for case in mm["rejected"]:
        with pytest.raises(_lib.SkError):
            gpu.read_matrix_market(case["text"].encode())
    for case in mm["write"]:
        Ad = gpu.Device_matrix(csr_from_entries(tuple(case["shape"]), case["entries"]))
        out = tmp_path / "w.mtx"
        gpu.write_matrix_market(Ad, out)
        assert out.read_bytes() == case["text"].encode(), case["source"]


def test_malformed_input_is_an_error(gpu_lib, tmp_path):
    """What the reference leaves undefined is an error here: fewer entry
    lines than announced, an index outside the shape, a line that is not
    'row col value'; and a side of 1 is rejected as the reference does."""
    head = "%%MatrixMarket matrix coordinate real general\n"
    for body in ("3 3 4\n1 1 1.0\n2 2 2.0\n", "3 3 1\n4 1 1.0\n", "3 3 1\n0 1 1.0\n", "3 3 2\n1 1 1.0\n% x\n",
                 "3 3 1\n1 x 1.0\n", "1 3 1\n1 1 1.0\n", "", "% only a comment\n"):
        with pytest.raises(_lib.SkError):
            gpu.read_matrix_market((head + body).encode())
    with pytest.raises(_lib.SkError):
        gpu.read_matrix_market(tmp_path / "missing.mtx")


def test_full_size_round_trip(gpu_lib, oracle, tmp_path):
    """The 128^3 7-point Laplacian (14.6M entries) written with 17
    significant digits and read back gives the same CSR arrays; a seeded
    1M x 1M symmetric file (lower triangle, with duplicates) reads as the
    oracle reads it."""
    A = matgen.laplacian_3d_dirichlet(128)
    path = tmp_path / "lap.mtx"
    gpu.write_matrix_market(gpu.Device_matrix(A), path, precision=17)
    B = gpu.read_matrix_market(path).to_host()
    for f in ("row_ptr", "col_ind", "values"):
        assert _same_bits(getattr(B, f)(), getattr(A, f)()), f
    rng = np.random.default_rng(9)
    n, k = 1_000_000, 3_000_000
    r, c = rng.integers(1, n + 1, k), rng.integers(1, n + 1, k)
    r, c = np.maximum(r, c), np.minimum(r, c)
    r[-1000:], c[-1000:] = r[:1000], c[:1000]
    v = rng.standard_normal(k)
    body = "\n".join(f"{a} {b} {x:.17g}" for a, b, x in zip(r.tolist(), c.tolist(), v.tolist()))
    text = f"%%MatrixMarket matrix coordinate real symmetric\n{n} {n} {k}\n{body}\n".encode()
    G = gpu.read_matrix_market(text).to_host()
    O = oracle.mm_read(text)
    for f in ("row_ptr", "col_ind", "values"):
        assert _same_bits(getattr(G, f)(), getattr(O, f)()), f
