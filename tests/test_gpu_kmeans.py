"""GPU parity of the KMeans initialisation (VlGMMKMeans, vl/gmm.c:1315-1370)
through the C-ABI against VLFeat's own results (golden vectors from
tests/golden/make_golden.py).

Bit-exact: the k-means assignment of every row (the one-hot posteriors that
vl_gmm_init_with_kmeans leaves) and the generator's next draw after the
initialisation (the number of random draws: seeding shuffle, kd-tree builds,
restarts).  Within tolerance: the parameters of the one-hot M-step (the
library's M-step sums in another order than the reference's: float 2e-5,
double 1e-10 relative; float covariances 1e-4, because this M-step starts from
zero means (vl/gmm.c:1326-1328), so the variance is E[x^2] - mean^2 and both
implementations' float rounding is amplified by mean^2 / variance, about 125
on the one-dimensional case) and five EM iterations after the initialisation
(the bounds of the other EM tests: float 2e-4, double 1e-9)."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from conftest import rel_err

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_golden import KMEANS_CASES, kmeans_data  # noqa: E402

pytestmark = pytest.mark.gpu

DT = {"f": np.float32, "d": np.float64}
TOL = {"f": 2e-5, "d": 1e-10}
TOL_COVS = {"f": 1e-4, "d": 1e-10}
EM_TOL = {"f": 2e-4, "d": 1e-9}
CASES = [(n, t) for n, tags in KMEANS_CASES.items() for t in tags]


@pytest.fixture(autouse=True)
def exact_mode(vl):
    vl.set_precision("exact")
    yield


def _lanes_match(vl, golden):
    """The fixtures' distances follow the SIMD kernel the reference picked on
    the fixture host; the library picks by the same rule here."""
    L = vl.lib()
    ours = 8 if L.vl_cpu_has_avx() else (4 if L.vl_cpu_has_sse2() else 1)
    return ours == int(golden["rand_lanes"])


def _init(vl, x, K, seed):
    m = vl.GMM(x.shape[1], K, x.dtype.type)
    m.set_covariance_lower_bound(1e-4)
    vl.rand_seed(seed)
    vl._clear()
    vl.lib().vl_gmm_init_with_kmeans(m._h, x.ctypes.data_as(C.c_void_p), x.shape[0], None)
    assert vl.lib().vl_get_last_error() == 0, vl.lib().vl_get_last_error_message()
    nxt = vl.rand_uint32()
    return m, nxt


@pytest.mark.parametrize("name,tag", CASES)
def test_kmeans_init_matches_reference(vl, golden, name, tag):
    if not _lanes_match(vl, golden):
        pytest.skip("this host's SIMD support differs from the fixture host's")
    x, K, seed = kmeans_data(name)
    x = np.ascontiguousarray(x.astype(DT[tag]))
    m, nxt = _init(vl, x, K, seed)
    post = m.posteriors
    assert post.shape == (x.shape[0], K)
    # One-hot rows: exactly one 1 per row.
    assert np.array_equal(post.sum(axis=1), np.ones(x.shape[0]))
    assign = np.argmax(post, axis=1)
    ref = golden[f"km_{name}_{tag}_assign"]
    assert np.array_equal(assign, ref), f"{int((assign != ref).sum())} rows assigned differently"
    assert nxt == int(golden[f"km_{name}_{tag}_next"])
    for k, got in (("means", m.means), ("covs", m.covariances), ("priors", m.priors)):
        tol = TOL_COVS[tag] if k == "covs" else TOL[tag]
        assert rel_err(got, golden[f"km_{name}_{tag}_{k}"]) < tol, k


@pytest.mark.parametrize("name,tag", [("small", "f"), ("small", "d"), ("mix", "f"), ("mix", "d")])
def test_kmeans_init_then_em(vl, golden, name, tag):
    """vl_gmm_cluster with VlGMMKMeans and five EM iterations."""
    if not _lanes_match(vl, golden):
        pytest.skip("this host's SIMD support differs from the fixture host's")
    x, K, seed = kmeans_data(name)
    x = np.ascontiguousarray(x.astype(DT[tag]))
    m = vl.GMM(x.shape[1], K, x.dtype.type)
    m.set_initialization("kmeans")
    m.set_max_num_iterations(5)
    m.set_covariance_lower_bound(1e-4)
    vl.rand_seed(seed)
    ll = m.cluster(x)
    tol = EM_TOL[tag]
    ref_ll = float(golden[f"km_{name}_{tag}_t5_ll"])
    assert abs(ll - ref_ll) <= tol * abs(ref_ll)
    assert rel_err(m.means, golden[f"km_{name}_{tag}_t5_means"]) < tol
    assert rel_err(m.covariances, golden[f"km_{name}_{tag}_t5_covs"]) < tol
    assert rel_err(m.priors, golden[f"km_{name}_{tag}_t5_priors"]) < tol


def test_kmeans_object_lifecycle(vl, golden):
    """The GMM creates its k-means object on first use and keeps it
    (vl/gmm.c:1336-1356); a second initialisation reuses it and draws afresh
    from the generator; vl_gmm_reset drops it; an object from elsewhere is
    refused with an error."""
    L = vl.lib()
    x, K, seed = kmeans_data("small")
    x = np.ascontiguousarray(x.astype(np.float32))
    m = vl.GMM(x.shape[1], K, np.float32)
    assert not L.vl_gmm_get_kmeans_init_object(m._h)
    vl.rand_seed(seed)
    vl._clear()
    L.vl_gmm_init_with_kmeans(m._h, x.ctypes.data_as(C.c_void_p), x.shape[0], None)
    assert L.vl_get_last_error() == 0
    obj = L.vl_gmm_get_kmeans_init_object(m._h)
    assert obj
    a1 = np.argmax(m.posteriors, axis=1)
    L.vl_gmm_init_with_kmeans(m._h, x.ctypes.data_as(C.c_void_p), x.shape[0], None)
    assert L.vl_gmm_get_kmeans_init_object(m._h) == obj
    assert L.vl_get_last_error() == 0
    if _lanes_match(vl, golden):
        assert np.array_equal(a1, golden["km_small_f_assign"])
    L.vl_gmm_reset(m._h)
    assert not L.vl_gmm_get_kmeans_init_object(m._h)
    foreign = C.create_string_buffer(64)
    L.vl_gmm_set_kmeans_init_object(m._h, C.cast(foreign, C.c_void_p))
    L.vl_gmm_init_with_kmeans(m._h, x.ctypes.data_as(C.c_void_p), x.shape[0], None)
    assert L.vl_get_last_error() != 0
    L.vl_gmm_set_kmeans_init_object(m._h, None)


def test_kmeans_repetitions(vl):
    """Two repetitions of vl_gmm_cluster with KMeans initialisation: each
    repetition initialises afresh from the generator; the best
    log-likelihood is kept (vl/gmm.c:1583-1640)."""
    x, K, seed = kmeans_data("mix")
    x = np.ascontiguousarray(x.astype(np.float32))
    ll = []
    for reps in (1, 2):
        m = vl.GMM(x.shape[1], K, np.float32)
        m.set_initialization("kmeans")
        m.set_max_num_iterations(3)
        m.set_num_repetitions(reps)
        vl.rand_seed(seed)
        ll.append(m.cluster(x))
        assert vl.lib().vl_get_last_error() == 0
    assert ll[1] >= ll[0]
