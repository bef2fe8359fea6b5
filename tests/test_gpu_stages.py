"""Parity of the stage compositions (navier.f90, transeq.f90, poisson.f90,
time_integrators.f90, mom.f90) against the CPU oracle, plus the
size-independent properties checked at 512^3."""
import numpy as np
import pytest

from conftest import rel_err, seeded_field

pytestmark = pytest.mark.gpu

# (18, 12, 10): x not a multiple of 4, so the fused stage kernels step aside
# for the one-launch-per-operator composition.
SHAPES = [(16, 16, 16), (24, 20, 12), (32, 32, 32), (18, 12, 10)]
LEN = (2 * np.pi, 1.5, 3.0)


def fields(shape, seeds=(1, 2, 3)):
    return [seeded_field(shape, s, lengths=LEN, noise=1e-2) for s in seeds]


def ctx_for(shape, prec="f64"):
    from x3div_b200 import Context
    return Context(*shape, lengths=LEN, precision=prec)


@pytest.mark.parametrize("shape", SHAPES)
def test_poisson(oracle, torch_cuda, shape):
    from x3div_b200 import to_device, to_host
    ctx = ctx_for(shape)
    rhs = seeded_field(shape, 21, kind="rand", lengths=LEN, noise=0)
    d = to_device(rhs)
    ctx.poisson(d)
    ctx.sync()
    assert rel_err(to_host(d), oracle.poisson(rhs, *LEN)) < 1e-12
    ctx.close()


# z lengths of every radix pattern of the fused z-transform kernel (8s, 4, 2,
# 3s; one to four tiles of x modes, a last tile of one mode) and two that
# take the 3-D cuFFT path (nz = 40 = 8 * 5, and nz = 2048, above the longest
# fused transform)
@pytest.mark.parametrize("shape", [(16, 10, 8), (30, 12, 12), (34, 8, 48), (20, 8, 96), (14, 8, 192),
                                   (8, 8, 384), (8, 8, 768), (10, 8, 1024), (12, 10, 40), (8, 12, 2048)])
def test_poisson_z_lengths(oracle, torch_cuda, shape):
    from x3div_b200 import to_device, to_host
    ctx = ctx_for(shape)
    rhs = seeded_field(shape, 23, kind="rand", lengths=LEN, noise=0)
    d = to_device(rhs)
    ctx.poisson(d)
    ctx.sync()
    assert rel_err(to_host(d), oracle.poisson(rhs, *LEN)) < 1e-12, shape
    ctx.close()


# x lengths of every own x transform (nx / 2 from 8 to 1024) with y extents
# that mostly leave a partial last tile of rows (4 rows a tile), each solved
# through the own x transforms (the default) and through cuFFT's 2-D (x, y)
# transforms (stage choice poisson_x = 0).
@pytest.mark.parametrize("shape", [(16, 10, 8), (24, 9, 12), (48, 9, 16), (96, 9, 24), (192, 10, 32),
                                   (384, 12, 48), (768, 10, 16), (1024, 9, 8), (1536, 9, 8), (2048, 9, 12),
                                   (512, 33, 64), (64, 64, 64), (128, 20, 96), (256, 17, 128), (16, 12, 768),
                                   (32, 9, 1024)])
def test_poisson_own_x_transforms(oracle, torch_cuda, shape):
    from x3div_b200 import to_device, to_host
    rhs = seeded_field(shape, 31, kind="rand", lengths=LEN, noise=0)
    ref = oracle.poisson(rhs, *LEN)
    outs = []
    for choice in (-1, 0):
        ctx = ctx_for(shape)
        ctx.set_stage_choice("poisson_x", choice)
        d = to_device(rhs)
        n0 = ctx.launch_count()
        ctx.poisson(d)
        ctx.sync()
        # own x transforms: x forward, z solve, x inverse (the y transforms are cuFFT's)
        assert ctx.launch_count() - n0 == (3 if choice == -1 else 1), (shape, choice)
        outs.append(to_host(d))
        assert rel_err(outs[-1], ref) < 1e-12, (shape, choice)
        ctx.close()
    assert rel_err(outs[0], outs[1]) < 1e-13, shape


def test_poisson_x_choice_is_checked(torch_cuda):
    from x3div_b200 import X3DError
    ctx = ctx_for((16, 16, 16))
    with pytest.raises(X3DError):
        ctx.set_stage_choice("poisson_x", 2)
    ctx.set_stage_choice("poisson_x", 0)
    ctx.set_stage_choice("poisson_x", -1)
    ctx.close()


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_divergence_gradp_momentum(oracle, torch_cuda, shape, prec):
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    ctx = ctx_for(shape, prec)
    dt = torch.float64 if prec == "f64" else torch.float32
    # FP32: each interpolation alone is ~6e-6 (cond ~ 99 for alpha = 0.49,
    # times FP32 rounding of its LU factors); a stage chains three operators.
    tol = 1e-12 if prec == "f64" else 1e-4
    u, v, w = fields(shape)
    ud, vd, wd = (to_device(a, dt) for a in (u, v, w))
    uh, vh, wh = (to_host(a).astype(np.float64) for a in (ud, vd, wd))
    dx, dy, dz = ctx.dx, ctx.dy, ctx.dz
    # divergence (pp3 is FP64 in both precisions)
    pp3 = torch.empty(shape[::-1], dtype=torch.float64, device="cuda")
    ctx.divergence(pp3, ud, vd, wd)
    ctx.sync()
    ref_div = oracle.divergence(uh, vh, wh, dx, dy, dz)
    assert rel_err(to_host(pp3), ref_div) < tol
    # gradp from an FP64 pressure
    px, py, pz = (torch.empty_like(ud) for _ in range(3))
    p_h = seeded_field(shape, 30, kind="rand", lengths=LEN, noise=0)
    p_d = to_device(p_h)
    n0 = ctx.launch_count()
    ctx.gradp(px, py, pz, p_d)
    ctx.sync()
    # three fused stages (x lines of 16-byte vectors); an FP32 step stages
    # the FP64 pressure in its z launch rather than converting it first
    if shape[0] * (8 if prec == "f64" else 4) % 16 == 0:
        assert ctx.launch_count() - n0 == 3, ctx.launch_count() - n0
    rp = oracle.gradp(p_h, dx, dy, dz)
    for got, ref in zip((px, py, pz), rp):
        assert rel_err(to_host(got), ref) < tol
    # momentum_rhs_eq
    du = [torch.empty_like(ud) for _ in range(3)]
    ctx.momentum_rhs_eq(*du, ud, vd, wd)
    ctx.sync()
    ref_du = oracle.momentum_rhs(uh, vh, wh, dx, dy, dz)
    for got, ref in zip(du, ref_du):
        assert rel_err(to_host(got), ref) < tol
    ctx.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_euler_steps_match_oracle(oracle, torch_cuda, prec):
    """Ten x3div timesteps (dt = 1e-3) against the oracle; the divergence after
    each projection is round-off in FP64."""
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    shape = (32, 24, 16)
    ctx = ctx_for(shape, prec)
    dt_ = torch.float64 if prec == "f64" else torch.float32
    u, v, w = fields(shape, (5, 6, 7))
    U = [to_device(a, dt_) for a in (u, v, w)]
    ref = [to_host(a).astype(np.float64) for a in U]
    du = [torch.empty_like(U[0]) for _ in range(3)]
    pg = [torch.empty_like(U[0]) for _ in range(3)]
    pp3 = torch.empty(shape[::-1], dtype=torch.float64, device="cuda")
    for _ in range(10):
        ctx.euler_step(*U, *du, pp3, *pg, 1e-3)
        oracle.euler_step(*ref, 1e-3, lengths=LEN)
    ctx.sync()
    tol = 1e-11 if prec == "f64" else 1e-4
    for got, r in zip(U, ref):
        assert rel_err(to_host(got), r) < tol
    if prec == "f64":
        div = torch.empty_like(pp3)
        ctx.divergence(div, *U)
        mx, mean = ctx.div_stats(div)
        assert mx < 1e-10
    ctx.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_autotuned_euler_steps_match_oracle(oracle, torch_cuda, prec):
    """After x3d_autotune (which also picks a kernel for each fused Euler
    stage, timing them on scratch fields), three timesteps still match the
    oracle, and the tuning left the caller's fields untouched."""
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    shape = (64, 48, 32)
    ctx = ctx_for(shape, prec)
    dt_ = torch.float64 if prec == "f64" else torch.float32
    u, v, w = fields(shape, (8, 9, 10))
    U = [to_device(a, dt_) for a in (u, v, w)]
    before = [to_host(a).copy(order="F") for a in U]
    ctx.autotune(1)
    for a, b in zip(U, before):
        assert np.array_equal(to_host(a), b)
    ref = [b.astype(np.float64) for b in before]
    du = [torch.empty_like(U[0]) for _ in range(3)]
    pg = [torch.empty_like(U[0]) for _ in range(3)]
    pp3 = torch.empty(shape[::-1], dtype=torch.float64, device="cuda")
    for _ in range(3):
        ctx.euler_step(*U, *du, pp3, *pg, 1e-3)
        oracle.euler_step(*ref, 1e-3, lengths=LEN)
    ctx.sync()
    tol = 1e-11 if prec == "f64" else 1e-4
    for got, r in zip(U, ref):
        assert rel_err(to_host(got), r) < tol
    ctx.set_kernel(-1)
    ctx.close()


# Every stage that can run as several launches, forced on: the momentum
# stages as two launches of two staged fields, the others as one launch per
# disjoint set of staged inputs.
SPLIT_FORMS = {"transeq_x.split": 1, "transeq_y.split": 1, "transeq_z.split": 1, "div_x.parts": 3,
               "div_y.parts": 2, "gradp_y.parts": 2, "gradp_x.parts": 3, "gradp_x_cor.parts": 3}


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(64, 48, 32), (36, 60, 62)])
def test_split_stage_forms_match_the_one_launch_stages(oracle, torch_cuda, prec, shape):
    """With every split form pinned (x3d_ctx_set_stage_choice), three Euler
    steps equal those of the one-launch stages bit for bit (the same kernel
    configuration and the same arithmetic per output; the z momentum stage
    updates u in place, so its launch that writes u_z runs last) and match
    the oracle; the split context launched more kernels."""
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    one, split = ctx_for(shape, prec), ctx_for(shape, prec)
    for k, v in SPLIT_FORMS.items():
        split.set_stage_choice(k, v)
        assert split.autotune_stage_choice(k) == v
    dt_ = torch.float64 if prec == "f64" else torch.float32
    U = [to_device(a, dt_) for a in fields(shape, (14, 15, 16))]
    V = [a.clone() for a in U]
    ref = [to_host(a).astype(np.float64) for a in U]
    du = [torch.empty_like(U[0]) for _ in range(3)]
    pg = [torch.empty_like(U[0]) for _ in range(3)]
    dv = [torch.empty_like(U[0]) for _ in range(3)]
    pv = [torch.empty_like(U[0]) for _ in range(3)]
    pp3 = torch.empty(shape[::-1], dtype=torch.float64, device="cuda")
    pq = torch.empty_like(pp3)
    n1, n2 = one.launch_count(), split.launch_count()
    for _ in range(3):
        one.euler_step(*U, *du, pp3, *pg, 1e-3)
        split.euler_step(*V, *dv, pq, *pv, 1e-3)
        oracle.euler_step(*ref, 1e-3, lengths=LEN)
    one.sync()
    split.sync()
    assert split.launch_count() - n2 > one.launch_count() - n1
    tol = 1e-11 if prec == "f64" else 1e-4
    for a, b, r in zip(U, V, ref):
        assert torch.equal(a, b)
        assert rel_err(to_host(a), r) < tol
    assert torch.equal(pp3, pq)
    with pytest.raises(Exception):
        split.set_stage_choice("transeq_x.split", 2)
    split.set_stage_choice("transeq_x.split", -1)
    assert split.autotune_stage_choice("transeq_x.split") == -1
    one.close()
    split.close()


def test_reference_test_mode(oracle, torch_cuda):
    """test_du/dv/dw on the reference vel field (src/mom.f90) match the oracle's RMS."""
    torch = torch_cuda
    from x3div_b200 import Context, to_host
    n = 64
    ctx = Context(n, n, n)  # reference box: xlx = yly = zlz = 1
    U = [torch.empty(n, n, n, dtype=torch.float64, device="cuda") for _ in range(3)]
    ctx.vel(*U)
    ctx.sync()
    ref = oracle.vel(n, n, n)
    for got, r in zip(U, ref):
        assert rel_err(to_host(got), r) < 1e-14
    names = ("derx", "dery", "derz")
    for which in range(3):
        t = torch.empty_like(U[0])
        fn = getattr(ctx, names[which])
        if which == 1:
            fn(t, U[which], ctx.op("dery"), None, n, n, n)
        else:
            fn(t, U[which], ctx.op(names[which]), n, n, n)
        rms = ctx.test_rms(which, t)
        ref_rms = oracle.test_rms(which, oracle.apply("der", which, ref[which], 1.0 / n))
        assert abs(rms - ref_rms) < 1e-6 * ref_rms
    ctx.close()


def test_transposes_are_layout_copies(torch_cuda):
    torch = torch_cuda
    from x3div_b200 import Context
    ctx = Context(16, 12, 8, precision="f32")
    a = torch.randn(8, 12, 16, device="cuda")
    b = torch.empty_like(a)
    for name in ("x_to_y", "y_to_z", "z_to_y", "y_to_x"):
        b.zero_()
        getattr(ctx, "transpose_" + name)(a, b)
        ctx.sync()
        assert torch.equal(a, b)
    c = torch.randn(8, 12, 32, device="cuda")  # complex: twice the bytes
    d = torch.empty_like(c)
    ctx.transpose_x_to_y(c, d, is_complex=True)
    ctx.sync()
    assert torch.equal(c, d)
    ctx.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_512_selected_ops(oracle, torch_cuda, prec):
    """Full-size (512^3) parity for one operator per kernel family and
    direction, against the oracle on the same input."""
    torch = torch_cuda
    from x3div_b200 import Context, to_device, to_host
    n = 512
    ctx = Context(n, n, n, lengths=(2 * np.pi,) * 3, precision=prec)
    dt = torch.float64 if prec == "f64" else torch.float32
    u_h = seeded_field((n, n, n), 512, noise=1e-3)
    u = to_device(u_h, dt)
    del u_h
    used = to_host(u).astype(np.float64)
    tol = 1e-12 if prec == "f64" else 1e-5
    t = torch.empty_like(u)
    cases = [("derx", "derx", "der", 0), ("interyvp", "intyvp", "intvp", 1), ("derzz", "derzz", "der2", 2)]
    for routine, opn, kind, direction in cases:
        if routine == "interyvp":
            ctx.interyvp(t, u, ctx.op(opn), n, n, n, n)
        else:
            getattr(ctx, routine)(t, u, ctx.op(opn), n, n, n)
        ctx.sync()
        ref = oracle.apply(kind, direction, used, 2 * np.pi / n)
        assert rel_err(to_host(t), ref) < tol, (routine, prec)
    ctx.close()


@pytest.mark.parametrize("cfg", [6, 12, 13, 14, 15])
@pytest.mark.parametrize("shape", [(64, 48, 32), (36, 60, 62)])
def test_forced_stage_configurations_match_oracle(oracle, torch_cuda, cfg, shape):
    """Three FP32-mixed timesteps with every fused stage forced onto one kernel
    configuration: 6 (one line per thread), 12-15 (two x-adjacent y/z lines
    per thread in packed FP32 registers), whose transeq, divergence and gradp
    launches take every flush form (plain, du += ..., u = u + dt du, FP64 pp3,
    u -= grad p).  Stages that a configuration cannot take fall back."""
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    ctx = ctx_for(shape, "f32")
    ctx.set_kernel(cfg)
    U = [to_device(a, torch.float32) for a in fields(shape, (11, 12, 13))]
    ref = [to_host(a).astype(np.float64) for a in U]
    du = [torch.empty_like(U[0]) for _ in range(3)]
    pg = [torch.empty_like(U[0]) for _ in range(3)]
    pp3 = torch.empty(shape[::-1], dtype=torch.float64, device="cuda")
    for _ in range(3):
        ctx.euler_step(*U, *du, pp3, *pg, 1e-3)
        oracle.euler_step(*ref, 1e-3, lengths=LEN)
    ctx.sync()
    for got, r in zip(U, ref):
        assert rel_err(to_host(got), r) < 1e-4, cfg
    ctx.set_kernel(-1)
    ctx.close()
