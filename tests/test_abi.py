"""CPU tests of the drop-in boundary: the library loads, exports every symbol
the public headers declare, and reports failures through VLFeat's
last-error channel instead of aborting (no kernel runs here)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADERS = ["include/vl/generic.h", "include/vl/random.h", "include/vl/gmm.h", "include/vl/fisher.h",
           "include/vl/vlad.h", "include/vlb200.h"]


def declared_symbols():
    names = set()
    for h in HEADERS:
        src = open(os.path.join(ROOT, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"VL_EXPORT[^;(]*?\b(\w+)\s*\(", src):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def libpath():
    from vlfeat_b200 import build
    return build.build()


def test_header_declarations_found():
    names = declared_symbols()
    assert {"vl_gmm_new", "vl_gmm_cluster", "vl_fisher_encode", "vl_get_gmm_data_posteriors_f",
            "vlb200_fisher_encode_batch_device", "vl_vlad_encode", "vl_rand_uint32",
            "vlb200_vlad_encode_batch_device"} <= names
    assert len(names) > 60


def test_exports_every_declared_symbol(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = declared_symbols() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_loads_and_binds(libpath):
    from vlfeat_b200 import capi
    L = capi.lib()
    assert L.vl_get_version_string()
    assert L.vlb200_version().startswith(b"vlfeat-b200")


def test_model_state_without_gpu(libpath):
    """Object lifecycle, setters and getters are host-only and match the
    reference defaults (vl/gmm.c:353-382)."""
    import numpy as np
    from vlfeat_b200 import capi
    g = capi.GMM(5, 3)
    L = capi.lib()
    assert L.vl_gmm_get_max_num_iterations(g._h) == 50
    assert L.vl_gmm_get_num_repetitions(g._h) == 1
    assert L.vl_gmm_get_initialization(g._h) == capi.INIT_RAND
    lb = np.ctypeslib.as_array(C.cast(L.vl_gmm_get_covariance_lower_bounds(g._h),
                                      C.POINTER(C.c_double)), shape=(5,))
    assert np.all(lb == 1e-4)
    g.set_means(np.arange(15, dtype=np.float32).reshape(3, 5))
    assert np.array_equal(g.means, np.arange(15, dtype=np.float32).reshape(3, 5))
    g.set_covariance_lower_bound(0.5)
    assert np.all(np.ctypeslib.as_array(C.cast(L.vl_gmm_get_covariance_lower_bounds(g._h),
                                               C.POINTER(C.c_double)), shape=(5,)) == 0.5)


def test_bad_arguments_set_last_error(libpath):
    import numpy as np
    from vlfeat_b200 import capi
    L = capi.lib()
    enc = np.zeros(4, np.float32)
    nt = L.vl_fisher_encode(enc.ctypes.data_as(C.c_void_p), 7, None, 1, 1, None, None, None, 0, 0)
    assert nt == 0 and L.vl_get_last_error() == 3  # VL_ERR_BAD_ARG
    assert L.vlb200_set_precision(99) == 3


def test_without_gpu_reports_error(libpath):
    import numpy as np
    from vlfeat_b200 import capi
    if capi.device_ok():
        pytest.skip("a GPU is present; the failure path is exercised only without one")
    with pytest.raises(capi.VLError):
        capi.fisher_encode(np.zeros((3, 2), np.float32), np.zeros((1, 2), np.float32),
                           np.ones((1, 2), np.float32), np.ones(1, np.float32))


def test_fisher_plan_argument_checks(libpath):
    """The plan's argument checks run on the host before any device call:
    precision EXACT (the plan is the tensor-core encoder), an unsupported
    dimension and decreasing offsets return NULL with VL_ERR_BAD_ARG."""
    import numpy as np
    from vlfeat_b200 import capi
    L = capi.lib()
    offs = np.array([0, 10, 25], np.int64)
    assert not L.vlb200_fisher_plan_new(80, 256, capi._np_ptr(offs), 2, 0, 1)  # EXACT
    assert L.vl_get_last_error() == 3
    assert not L.vlb200_fisher_plan_new(96, 256, capi._np_ptr(offs), 2, 0, 3)  # D = 96
    assert L.vl_get_last_error() == 3
    bad = np.array([0, 10, 5], np.int64)
    assert not L.vlb200_fisher_plan_new(80, 256, capi._np_ptr(bad), 2, 0, 3)
    assert L.vl_get_last_error() == 3
    assert L.vlb200_fisher_plan_launch(None, None) == 3


def test_library_rng_matches_reference(libpath, golden):
    """The library's per-thread MT19937 (vl_get_rand, vl_rand_seed,
    vl_rand_uint32; host code) draws the reference's sequence."""
    from vlfeat_b200 import capi
    capi.rand_seed(int(golden["rng_seed"]))
    seq = [capi.rand_uint32() for _ in range(len(golden["rng_seq"]))]
    assert seq == [int(v) for v in golden["rng_seq"]]


def test_vlad_argument_checks(libpath):
    """VLAD's argument checks run before any device call: an unknown data
    type, decreasing offsets and a dimension above 1024 fail with
    VL_ERR_BAD_ARG through the last-error channel."""
    import numpy as np
    from vlfeat_b200 import capi
    L = capi.lib()
    enc = np.zeros(4, np.float32)
    L.vl_set_last_error(0, b"")
    L.vl_vlad_encode(enc.ctypes.data_as(C.c_void_p), 7, None, 2, 2, None, 0, None, 0)
    assert L.vl_get_last_error() == 3
    bad = np.array([0, 10, 5], np.int64)
    assert L.vlb200_vlad_encode_batch_device(None, 1, None, 8, 4, None, None, capi._np_ptr(bad), 2, 0,
                                             C.c_void_p(1)) == 3
    assert L.vlb200_vlad_encode_batch_device(None, 9, None, 8, 4, None, None, capi._np_ptr(bad[:1]), 0, 0,
                                             C.c_void_p(1)) == 3
    offs = np.array([0, 10], np.int64)
    assert L.vlb200_vlad_encode_batch_device(None, 1, None, 1025, 4, None, None, capi._np_ptr(offs), 1, 0,
                                             C.c_void_p(1)) == 3


def test_pca_argument_checks(libpath):
    """Dimensions above 128 and frames without image sizes fail with
    VL_ERR_BAD_ARG before any device work."""
    import numpy as np
    from vlfeat_b200 import capi
    L = capi.lib()
    offs = np.array([0, 10], np.int64)
    assert L.vlb200_pca_project_device(None, 80, None, 129, 10, None, None, 1, None, None, None, 0,
                                       C.c_void_p(1)) == 3
    assert L.vlb200_pca_project_device(None, 80, None, 128, 10, None, None, 1, C.c_void_p(16), None, None, 1,
                                       C.c_void_p(1)) == 3
    assert L.vlb200_pca_learn_device(None, None, 81, None, 80, 10, 0, 0.0, None, C.c_void_p(1)) == 3


def test_precision_default_from_environment():
    """The process-wide mode starts as EXACT; VLB200_PRECISION=fp32 or bf16 in
    the environment selects another mode when the library is loaded."""
    import os
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); from vlfeat_b200 import capi; "
            "print(capi.get_precision())" % ROOT)
    for env, want in ((None, 1), ("fp32", 2), ("bf16", 3), ("bogus", 1)):
        e = dict(os.environ)
        e.pop("VLB200_PRECISION", None)
        if env:
            e["VLB200_PRECISION"] = env
        out = subprocess.run([sys.executable, "-c", code], env=e, capture_output=True, text=True, check=True)
        assert int(out.stdout.strip()) == want, (env, out.stdout)
