"""Parity of exactly what bench.py times, at the size it times it.

- The 512^3 derivative sweep: after x3d_autotune(6), the six operator
  families of one field and one direction go through x3d_apply_batch as one
  six-output launch (the bench's grouping, so the launches run the
  configurations the autotuner picked for six-operator groups).  All 18
  family x direction outputs of one field are compared with the oracle on the
  same input (FP64 <= 1e-12, FP32-mixed <= 1e-5 normwise relative).
  Reference: src/x3d_derive.f90:111-152, 279-339, 503-558 and the periodic
  branches of src/x3d_staggered.f90:23-404, 408-883, 887-1383.
- A 256^3 Euler step after x3d_autotune(1), two steps at the bench's
  dt = 5e-4, against the oracle's step (src/xcompact3d.f90:80-95): FP64
  <= 1e-11, FP32-mixed <= 1e-4 (stage chains of three operators), normwise
  over the velocity vector (max over u, v, w of the error / max over u, v,
  w of the field).
- The batching workload: one box of each of the five shapes the 48 boxes are
  drawn from, 3 FP32 fields each (Taylor-Green + N(0, (1e-2)^2)), all 54
  applications per box in the persistent batch launch, run plainly and
  replayed from its CUDA graph, every output against the oracle (<= 1e-5).

Inputs are the bench's own seeded fields.  Each oracle application at 512^3
takes about a second on 16 host threads; the whole file runs in a few
minutes on one B200 box.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

FAMILIES = [("der", ("derx", "dery", "derz")), ("der2", ("derxx", "deryy", "derzz")),
            ("dervp", ("derxvp", "deryvp", "derzvp")), ("derpv", ("derxpv", "derypv", "derzpv")),
            ("intvp", ("intxvp", "intyvp", "intzvp")), ("intpv", ("intxpv", "intypv", "intzpv"))]
B48_SHAPES = [(96, 96, 96), (128, 256, 64), (200, 100, 150), (256, 256, 256), (64, 512, 64)]


def bench_field(n, seed):
    """The bench's input: Taylor-Green component seed % 3 + N(0, (1e-3)^2)
    on an n^3 box of side 2 pi, as a Fortran-ordered (nx, ny, nz) array."""
    from bench import tg_noise
    return np.asfortranarray(tg_noise(n, seed).transpose(2, 1, 0))


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_sweep_512_autotuned_six_operator_launches(oracle, torch_cuda, prec):
    torch = torch_cuda
    from x3div_b200 import Context, to_device, to_host
    n = 512
    ctx = Context(n, n, n, lengths=(2 * np.pi,) * 3, precision=prec)
    ctx.autotune(6)
    dt = torch.float32 if prec == "f32" else torch.float64
    tol = 1e-5 if prec == "f32" else 1e-12
    u = to_device(bench_field(n, 0), dt)
    used = to_host(u).astype(np.float64)  # exactly what the kernels read
    outs = [torch.full_like(u, float("nan")) for _ in range(6)]
    h = 2 * np.pi / n
    errs = {}
    for d in range(3):
        cfg = ctx.autotune_choice(d, 6)
        assert 0 <= cfg <= 20 and cfg != 16, (d, cfg)  # a chunked (fused multi-output) configuration
        c0 = ctx.launch_count()
        ctx.apply_batch([(ctx.op(names[d]), u, outs[k]) for k, (_, names) in enumerate(FAMILIES)])
        ctx.sync()
        assert ctx.launch_count() - c0 == 1  # the six operators in one launch
        assert ctx.last_kernel() == cfg
        for k, (kind, names) in enumerate(FAMILIES):
            ref = oracle.apply(kind, d, used, h)
            err = rel_err(to_host(outs[k]), ref)
            errs[names[d]] = err
            assert err < tol, (prec, names[d], cfg, err)
            del ref
    print(f"\n512^3 {prec} six-operator launches, max error {max(errs.values()):.3e}:", errs)
    ctx.close()


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_euler_256_autotuned_steps(oracle, torch_cuda, prec):
    torch = torch_cuda
    from x3div_b200 import Context, to_device, to_host
    n = 256
    L = (2 * np.pi,) * 3
    ctx = Context(n, n, n, lengths=L, precision=prec)
    ctx.autotune(1)
    dt_ = torch.float32 if prec == "f32" else torch.float64
    U = [to_device(bench_field(n, s), dt_) for s in range(3)]
    ref = [to_host(a).astype(np.float64) for a in U]
    du = [torch.empty_like(U[0]) for _ in range(3)]
    pg = [torch.empty_like(U[0]) for _ in range(3)]
    pp3 = torch.empty((n, n, n), dtype=torch.float64, device="cuda")
    for _ in range(2):
        ctx.euler_step(*U, *du, pp3, *pg, 5e-4)
        oracle.euler_step(*ref, 5e-4, lengths=L)
    ctx.sync()
    # normwise over the velocity vector: w starts as the noise alone (the
    # Taylor-Green w is 0), so its own max is ~200x below max|u|, and the
    # error the projection spreads into it from u and v is measured against
    # the field's magnitude, max over the three components
    tol = 1e-11 if prec == "f64" else 1e-4
    got = [to_host(a) for a in U]
    scale = max(np.abs(r).max() for r in ref)
    err = max(np.abs(g - r).max() for g, r in zip(got, ref)) / scale
    per = [rel_err(g, r) for g, r in zip(got, ref)]
    print(f"\n256^3 {prec} two Euler steps, error {err:.3e} (per component, own max: {per}), "
          f"stages {ctx.stage_choices()}")
    assert err < tol, (err, per)
    ctx.close()


def b48_fields(torch, i, b):
    """Field f of box i as bench.py's batching leg makes it (Taylor-Green +
    N(0, (1e-2)^2), FP32), as a contiguous (nz, ny, nx) CUDA tensor."""
    nx, ny, nz = b
    x = torch.arange(nx, device="cuda", dtype=torch.float64) * (2 * np.pi / nx)
    y = torch.arange(ny, device="cuda", dtype=torch.float64) * (2 * np.pi / ny)
    z = torch.arange(nz, device="cuda", dtype=torch.float64) * (2 * np.pi / nz)
    tg = [torch.cos(z)[:, None, None] * torch.cos(y)[None, :, None] * torch.sin(x)[None, None, :],
          -torch.cos(z)[:, None, None] * torch.sin(y)[None, :, None] * torch.cos(x)[None, None, :],
          torch.zeros(nz, ny, nx, device="cuda", dtype=torch.float64)]
    g = torch.Generator(device="cuda")
    out = []
    for f in range(3):
        g.manual_seed(1000 * i + f)
        out.append((tg[f] + 1e-2 * torch.randn(nz, ny, nx, device="cuda", dtype=torch.float64,
                                                generator=g)).to(torch.float32).contiguous())
    return out


def test_b48_every_box_shape(oracle, torch_cuda):
    torch = torch_cuda
    from x3div_b200 import Batch, to_host
    fields, outs, used = [], [], []
    for i, b in enumerate(B48_SHAPES):
        fs = b48_fields(torch, i, b)
        fields.append(fs)
        used.append([to_host(a).astype(np.float64) for a in fs])
        outs.append([[[torch.full_like(fs[0], float("nan")) for _ in range(6)] for _ in range(3)]
                     for _ in range(3)])
    batch = Batch(B48_SHAPES, precision="f32")
    batch.bind_sweep(fields, outs)
    batch.autotune()  # as the bench does: chunk length and tile width per shape
    info = batch.info()
    assert info["fallback_jobs"] == 0  # every job in the one persistent launch
    assert info["points"] == 54 * sum(b[0] * b[1] * b[2] for b in B48_SHAPES)

    def check():
        worst = 0.0
        for i, b in enumerate(B48_SHAPES):
            h = [2 * np.pi / v for v in b]
            for f in range(3):
                for d in range(3):
                    for k, (kind, _) in enumerate(FAMILIES):
                        err = rel_err(to_host(outs[i][f][d][k]), oracle.apply(kind, d, used[i][f], h[d]))
                        worst = max(worst, err)
                        assert err < 1e-5, (b, f, d, kind, err)
        return worst

    batch.run()
    batch.sync()
    w1 = check()
    for per_box in outs:
        for per_f in per_box:
            for per_d in per_f:
                for o in per_d:
                    o.fill_(float("nan"))
    batch.capture()
    batch.replay()
    batch.replay()
    batch.sync()
    w2 = check()
    choices = {b: [batch.choice(i, d) for d in range(3)] for i, b in enumerate(B48_SHAPES)}
    print(f"\nB48 shapes: max error {w1:.3e} (run), {w2:.3e} (graph replay), {info}, tuned {choices}")
    batch.close()
