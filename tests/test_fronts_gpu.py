"""Dense fronts through the factorization kernels (the supernode-update
microbenchmark's path): L, D and the Schur update L21 D L21^T of seeded
complex-symmetric fronts against an FP64 host LDL^T of the same blocks --
<= 1e-12 relative in complex128, <= 1e-5 in complex64 on the tensor cores."""
import numpy as np
import pytest
import torch

import aphi_b200 as ab
from aphi_b200 import fronts_bench as fb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(ab.PREC_FP64, 1e-12), (ab.PREC_FP32, 1e-5)])
def test_fronts_match_host_ldlt(precision, tol, cuda):
    rows, widths, rng = fb.front_sizes(24, seed=5, lo=32, hi=700)
    rows[0], widths[0] = 640, 160          # a front with several 128-column panels
    fr = ab.Fronts(rows, widths)
    panels = fb.make_panels(rows, widths, rng)
    flat = torch.from_numpy(fb.pack(fr, panels)).cuda().unsqueeze(0)
    f = ab.Factor(fr, precision, 1)
    assert f.factorize_fronts(flat)
    p, c = f.read_fronts(0)
    err = fb.errors(fr, panels, p.cpu().numpy(), c.cpu().numpy(), range(len(rows)))
    assert err["max_rel_err_L"] <= tol and err["max_rel_err_D"] <= tol and err["max_rel_err_schur"] <= tol, err


def test_fronts_refuse_solves(cuda):
    fr = ab.Fronts([64], [16])
    f = ab.Factor(fr, ab.PREC_FP64, 1)
    rng = np.random.default_rng(0)
    flat = torch.from_numpy(fb.pack(fr, fb.make_panels(fr.rows, fr.widths, rng))).cuda().unsqueeze(0)
    assert f.factorize_fronts(flat)
    with pytest.raises(ab.AphiError):
        f.solve(torch.zeros((1, fr.n), dtype=torch.complex128, device="cuda"))
