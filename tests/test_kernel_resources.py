"""Register budgets of the hot kernels, from the ptxas reports the build
writes (no GPU needed).  The measured speeds depend on them:

- the fused step, gathered and not listed (every storage type, Smagorinsky
  form and map form): at most 64 registers (4 blocks of 256 threads per SM)
  and no spills; with the fused stress output at most 64 registers and a
  few spilled words (16 bytes at most);
- the row-staged steps: one cell per thread at most 72 registers (three CTAs
  of 288 threads per SM) with at most two spilled words; two cells per thread
  (16-bit storage) at most 128 registers (three CTAs of 160 threads), no
  spills in the reference Smagorinsky form the benchmarks run and at most
  24 bytes in the others;
- the PSC map scatter without periodic images: at most 48 registers (five
  256-thread blocks per SM) and no spills;
- the DEM kernels (contacts, integration, the cooperative and the one-block
  single launches): no spills;
- the stream / moments, sums and stress kernels: no spills.
"""
import os
import re

import pytest

BUILD = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lbdem_taichi_b200", "_build")


def _resources():
    from lbdem_taichi_b200 import build as B
    B.build()   # no-op when the library is current
    out = {}
    for f in sorted(os.listdir(BUILD)):
        if not f.endswith(".ptxas.txt"):
            continue
        txt = open(os.path.join(BUILD, f)).read()
        for block in re.split(r"ptxas info\s+: Compiling entry function '", txt)[1:]:
            name = block.split("'")[0]
            regs = int(re.search(r"Used (\d+) registers", block).group(1))
            spill = int(re.search(r"(\d+) bytes spill stores", block).group(1))
            out[name] = (regs, spill)
    return out


@pytest.fixture(scope="module")
def res():
    r = _resources()
    assert r, "no ptxas reports"
    return r


def _match(res, pattern):
    got = {k: v for k, v in res.items() if re.search(pattern, k)}
    assert got, pattern
    return got


def test_fused_step(res):
    # k_psc_step<T, GATHER=1, SMAG, WRAP, LISTED=0, STRESS=0, LAGM>: the lagged state in the storage
    # type (LAGM 0) for every form, and in FP16 (LAGM 1) under FP32 storage
    got = _match(res, r"k_psc_stepI(f|6__half|13__nv_bfloat16)Lb1ELi[012]ELb[01]ELb0ELb0ELi[01]E")
    assert len(got) == 3 * 3 * 2 + 3 * 2
    bad = {k: v for k, v in got.items() if v[0] > 64 or v[1] > 0}
    assert not bad, bad


def test_fused_step_with_stress(res):
    # k_psc_step<T, GATHER=1, SMAG, WRAP, LISTED=0, STRESS=1, LAGM=2 (width read at run time)>
    got = _match(res, r"k_psc_stepI(f|6__half|13__nv_bfloat16)Lb1ELi[012]ELb[01]ELb0ELb1ELi2E")
    assert len(got) == 3 * 3 * 2
    bad = {k: v for k, v in got.items() if v[0] > 64 or v[1] > 16}
    assert not bad, bad


def test_row_staged_steps(res):
    one = _match(res, r"k_psc_step_rowsI")
    assert len(one) == 3 * 3 * 2
    assert all(r <= 72 and s <= 8 for r, s in one.values()), one
    two = _match(res, r"k_psc_step_rows2I")
    assert len(two) == 2 * 3 * 2
    assert all(r <= 128 and s <= 24 for r, s in two.values()), two
    ref = {k: v for k, v in two.items() if "Li1E" in k}
    assert ref and all(s == 0 for _, s in ref.values()), ref


def test_map_scatter(res):
    got = _match(res, r"k_map_scatterILb0E")
    assert all(r <= 48 and s == 0 for r, s in got.values()), got


@pytest.mark.parametrize("kernel", ["k_contacts", "k_integrate", "k_dem_coop", "k_dem_block", "k_bin"])
def test_dem_kernels(res, kernel):
    got = _match(res, kernel)
    assert all(s == 0 for _, s in got.values()), got


@pytest.mark.parametrize("kernel", ["k_stream_moments", "k_sums", "k_stress"])
def test_auxiliary_kernels(res, kernel):
    got = _match(res, kernel)
    assert all(s == 0 for _, s in got.values()), got
