"""Precision of the table storage forms against the FP64 oracle (the restatement of the
reference's arithmetic in double, oracle/), with the plain FP32 form beside them.

Run with -s to print the tables (the figures quoted in the design notes come from this test):

    python -m pytest tests/test_precision.py -m gpu -s

Bars (relative L2 against the FP64 oracle, written here, used below):
  * plain forms (c64, r32): <= 1e-5, the parity bar of the path (measured ~5e-7: FP32 summation);
  * float16 forms (cf16, rf16, power-of-two scaled): <= 8e-4;
  * bfloat16 forms (cbf16, rbf16): <= 6e-3;
  * the same bounds for the bf16 form run batched on the 129^2-footprint table.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import REL_L2_FP32, VIS_SEED, oracle_config
from tconvolve.workload import PROBLEMS, batch_sizes, normal_vis

pytestmark = pytest.mark.gpu

BOUNDS = {"c64": REL_L2_FP32, "r32": REL_L2_FP32, "cf16": 8e-4, "rf16": 8e-4, "cbf16": 6e-3, "rbf16": 6e-3}
FORMS = list(BOUNDS)


def test_precision_table_forms(tcv, orc, cuda_ok):
    """The 1024^2-grid, 9-plane, 5 arcsec problem (16000 samples, 45^2 footprints), N(0,1) data."""
    prob = PROBLEMS["c1"]
    vis = normal_vis(prob.n_data(), VIS_SEED)
    r = orc.run_plain(oracle_config(orc, prob), vis=vis, threads=8, want_f64=True)
    b = tcv.Benchmark(**prob.kwargs())
    b.init()
    b.set_data(vis)
    rows = []
    for form in FORMS:
        b.set_ctype(form)
        b.zero_grid()
        b.runGrid()
        b.runDegrid()
        g, o = b.grid(), b.outdata()
        e_grid, e_out = orc.rel_l2(g, r["grid64"]), orc.rel_l2(o, r["outdata64"])
        rows.append((form, tcv.lib().tcv_ctype_bytes(tcv.CTYPE_BY_NAME[form]), e_grid, e_out))
        assert e_grid <= BOUNDS[form] and e_out <= BOUNDS[form], (form, e_grid, e_out)
    b.close()
    print("\n| form | table bytes/entry | grid rel-L2 vs FP64 | degridded rel-L2 vs FP64 | bound |")
    print("|---|---|---|---|---|")
    for form, nb, eg, eo in rows:
        print(f"| {form} | {nb} | {eg:.2e} | {eo:.2e} | {BOUNDS[form]:.0e} |")
    # the plain FP32 result against FP64, beside the reduced forms: FP32 summation only
    assert rows[0][2] < 2e-6 and rows[0][3] < 2e-6


@pytest.mark.parametrize("form", ["rbf16", "r32"])
def test_precision_batched_form(tcv, orc, cuda_ok, form):
    """The bf16 (and plain) form run batched on the 33-plane, 129^2-footprint table: the two
    smallest jobs of the 64-job batch against the FP64 oracle."""
    import torch

    from tconvolve import raw
    from tconvolve.batch import Batch, make_problem

    sizes = batch_sizes(64, seed=0)
    small = sorted(range(len(sizes)), key=lambda j: sizes[j][0])[:2]
    sub = [sizes[j] for j in small]
    p = make_problem(sub, vis_seed=VIS_SEED)
    ct = tcv.CTYPE_BY_NAME[form]
    c, scale, _ = raw.convert_c(p["c64"], ct)
    grids = [torch.zeros(g * g, dtype=torch.complex64, device="cuda") for _, g in sub]
    bt = Batch(sub, grids, p["iu"], p["iv"], p["coff"], p["support"], p["c_len"], tuning=(16, 64, 0, 512))
    bt.grid(p["data"], c, ct, scale)
    out = torch.empty(p["total"], dtype=torch.complex64, device="cuda")
    bt.degrid(c, ct, out, scale)
    torch.cuda.synchronize()
    # FP64 oracle on each job's in-bounds samples, with the real FP64 table of the same geometry
    prob = PROBLEMS["c2"]
    _, c64_f64, support, _, _, _ = orc.init_c(oracle_config(orc, prob), want_f64=True)
    iu, iv, co, data = (p[k].cpu().numpy() for k in ("iu", "iv", "coff", "data"))
    at = 0
    for j, (n, g) in enumerate(sub):
        sl = slice(at, at + n)
        s = 2 * support + 1
        keep = (iu[sl] - support >= 0) & (iu[sl] - support + s <= g) & (iv[sl] >= 0) & (iv[sl] + s <= g)
        ref = np.zeros(g * g, np.complex128)
        orc.grid_f64(data[sl][keep].astype(np.complex128), support, c64_f64, co[sl][keep], iu[sl][keep],
                     iv[sl][keep], ref, g)
        ref_o = orc.degrid_f64(ref, g, support, c64_f64, co[sl][keep], iu[sl][keep], iv[sl][keep])
        e_grid = orc.rel_l2(grids[j].cpu().numpy(), ref)
        e_out = orc.rel_l2(out[sl].cpu().numpy()[keep], ref_o)
        print(f"\nbatched {form} job {small[j]} ({n} samples, {g}^2): grid rel-L2 {e_grid:.2e}, "
              f"degridded rel-L2 {e_out:.2e} vs FP64")
        assert e_grid <= BOUNDS[form] and e_out <= BOUNDS[form], (e_grid, e_out)
        at += n
