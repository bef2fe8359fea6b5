"""FP32-mixed precision against FP64, per operator, on band-limited fields.

The field holds every Fourier mode with 0 < |k| <= N/4 at amplitude |k|^(-5/3)
and random phases.  Each of the six operator families is applied along each
direction by an FP32 context and by an FP64 context to the same field (the
FP32 input rounded from the FP64 one); the FP64 result matches the oracle to
1e-12, so it stands in for the exact answer.  Bar: both the normwise maximum
relative error max|a - b| / max|b| and the RMS relative error
||a - b||_2 / ||b||_2 are <= 1e-5.
"""
import numpy as np
import pytest

from conftest import band_limited_field

pytestmark = pytest.mark.gpu

# (routine, operator instance, signature style) for each family and direction
FAMILIES = {
    "der": [("derx", "derx", "d"), ("dery", "dery", "dy"), ("derz", "derz", "d")],
    "der2": [("derxx", "derxx", "d"), ("deryy", "deryy", "d"), ("derzz", "derzz", "d")],
    "dervp": [("derxvp", "derxvp", "x"), ("deryvp", "deryvp", "yd"), ("derzvp", "derzvp", "z")],
    "derpv": [("derxpv", "derxpv", "x"), ("derypv", "derypv", "yd"), ("derzpv", "derzpv", "z")],
    "intvp": [("interxvp", "intxvp", "x"), ("interyvp", "intyvp", "y"), ("interzvp", "intzvp", "z")],
    "intpv": [("interxpv", "intxpv", "x"), ("interypv", "intypv", "y"), ("interzpv", "intzpv", "z")],
}


def _call(ctx, routine, style, t, u, op, n):
    fn = getattr(ctx, routine)
    if style == "d":
        fn(t, u, op, n, n, n)
    elif style == "dy":
        fn(t, u, op, None, n, n, n)
    elif style in ("x", "y", "z"):
        fn(t, u, op, n, n, n, n)
    elif style == "yd":
        fn(t, u, op, None, n, n, n, n)


@pytest.mark.parametrize("n", [128, 256])
def test_fp32_matches_fp64_per_operator(torch_cuda, n):
    torch = torch_cuda
    from x3div_b200 import Context, to_device
    u64 = band_limited_field(n, seed=5 + n)
    ctx32 = Context(n, n, n, lengths=(2 * np.pi,) * 3, precision="f32")
    ctx64 = Context(n, n, n, lengths=(2 * np.pi,) * 3, precision="f64")
    d32 = to_device(u64, torch.float32)
    d64 = to_device(u64, torch.float64)
    t32 = torch.empty_like(d32)
    t64 = torch.empty_like(d64)
    worst = {}
    for fam, rows in FAMILIES.items():
        for routine, opname, style in rows:
            _call(ctx32, routine, style, t32, d32, ctx32.op(opname), n)
            _call(ctx64, routine, style, t64, d64, ctx64.op(opname), n)
            torch.cuda.synchronize()
            a = t32.double()
            b = t64
            emax = ((a - b).abs().max() / b.abs().max()).item()
            erms = (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()
            worst[routine] = (emax, erms)
            assert emax <= 1e-5 and erms <= 1e-5, (routine, emax, erms)
    ctx32.close()
    ctx64.close()
