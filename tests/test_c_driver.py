"""The drop-in boundary from C: tests/c/gmm_fisher_drop_in.c, a client
program written against VLFeat's public C API in the manner of the
reference's src/test_gmm.c:23-191, is compiled against this library's
include/ headers and linked twice -- with VLFeat's own CPU library (built from
the reference's sources into oracle/_ref) and with the GPU library -- and the
two runs' outputs are compared (float and double, Custom and Rand
initialisations: EM parameters, log-likelihood, posteriors, the improved
Fisher vector and its term count, VLAD).  The CPU test pins that the headers
are source- and binary-compatible with VLFeat's library."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "c", "gmm_fisher_drop_in.c")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libvl_ref.so")
GPU_LIB = os.path.join(ROOT, "vlfeat_b200", "lib", "libvl.so")
N, D, K, NF = 1000, 3, 20, 2000
CASES = ["float custom", "float rand", "double custom", "double rand"]


def _build_and_run(lib, tmp_path, tag):
    exe = str(tmp_path / f"drop_in_{tag}")
    out = str(tmp_path / f"out_{tag}.bin")
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
                    "-o", exe, lib, f"-Wl,-rpath,{os.path.dirname(lib)}", "-lm"], check=True)
    subprocess.run([exe, out], check=True, timeout=600)
    return _parse(np.fromfile(out, dtype=np.float64))


def _parse(a):
    sizes = [("ll", 1), ("means", K * D), ("covs", K * D), ("priors", K), ("post", N * K),
             ("fv", 2 * K * D), ("nterms", 1), ("vlad", K * D)]
    per = sum(n for _, n in sizes)
    assert a.size == per * len(CASES)
    out, o = [], 0
    for _ in CASES:
        r = {}
        for name, n in sizes:
            r[name] = a[o:o + n]
            o += n
        out.append(r)
    return out


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_c_program_runs_against_vlfeat(tmp_path):
    if not os.path.exists(REF_LIB):
        pytest.skip("VLFeat's CPU library is not built (oracle/Makefile ref)")
    res = _build_and_run(REF_LIB, tmp_path, "ref")
    for name, r in zip(CASES, res):
        for k, v in r.items():
            assert np.all(np.isfinite(v)), (name, k)
        assert r["nterms"][0] > 0, name


@pytest.mark.gpu
def test_c_program_drop_in_matches_vlfeat(tmp_path):
    if not os.path.exists(REF_LIB):
        pytest.skip("VLFeat's CPU library is not built (oracle/Makefile ref)")
    ref = _build_and_run(REF_LIB, tmp_path, "ref")
    got = _build_and_run(GPU_LIB, tmp_path, "gpu")
    for name, g, r in zip(CASES, got, ref):
        dbl = name.startswith("double")
        tol = 1e-9 if dbl else 2e-5
        assert abs(g["ll"][0] - r["ll"][0]) <= tol * abs(r["ll"][0]), name
        for k in ("means", "covs", "priors", "fv"):
            assert _rel(g[k], r[k]) < tol, (name, k)
        assert _rel(g["post"], r["post"]) < (1e-9 if dbl else 5e-5), name
        assert abs(g["nterms"][0] - r["nterms"][0]) <= (0 if dbl else 2), name
        assert _rel(g["vlad"], r["vlad"]) < (1e-9 if dbl else 1e-4), name
