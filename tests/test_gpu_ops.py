"""Parity of every operator routine of the C ABI against the CPU oracle.

Bars (normwise relative error, max|gpu - oracle| / max|oracle|):
  FP64 context: <= 1e-12 against the oracle on the same FP64 input.
  FP32 context: <= 1e-5 against the oracle on the same (FP32-rounded) input,
                i.e. the arithmetic of the FP32 sweeps themselves.
Shapes cover the TMA/bulk fast paths (x a multiple of 4) and the generic path
(odd sizes), lines from 8 (the minimum) upward, and non-cubic boxes.
"""
import numpy as np
import pytest

from conftest import rel_err, seeded_field

pytestmark = pytest.mark.gpu

X, Y, Z = 0, 1, 2
KERNEL_CONFIGS = 21  # x3d_ctx_set_kernel: 0..15 and 17..20 chunked, 16 one thread per line

# (routine, operator instance, oracle kind, direction, signature style)
ROUTINES = [
    ("derx", "derx", "der", X, "d"), ("dery", "dery", "der", Y, "dy"), ("derz", "derz", "der", Z, "d"),
    ("derx", "derxp", "der", X, "d"), ("dery", "deryp", "der", Y, "dy"), ("derz", "derzp", "der", Z, "d"),
    ("derxx", "derxx", "der2", X, "d"), ("deryy", "deryy", "der2", Y, "d"), ("derzz", "derzz", "der2", Z, "d"),
    ("derxvp", "derxvp", "dervp", X, "vp"), ("interxvp", "intxvp", "intvp", X, "vp"),
    ("derxpv", "derxpv", "derpv", X, "pv"), ("interxpv", "intxpv", "intpv", X, "pv"),
    ("interyvp", "intyvp", "intvp", Y, "vp"), ("deryvp", "deryvp", "dervp", Y, "vpy"),
    ("interypv", "intypv", "intpv", Y, "pv"), ("derypv", "derypv", "derpv", Y, "pvy"),
    ("derzvp", "derzvp", "dervp", Z, "vp"), ("interzvp", "intzvp", "intvp", Z, "vp"),
    ("derzpv", "derzpv", "derpv", Z, "pv"), ("interzpv", "intzpv", "intpv", Z, "pv"),
]

SHAPES = [(8, 8, 8), (9, 10, 11), (16, 17, 18), (32, 24, 40), (64, 64, 64), (40, 36, 12), (100, 12, 20)]


def call(ctx, routine, style, t, u, op, shape):
    nx, ny, nz = shape
    fn = getattr(ctx, routine)
    if style == "d":
        fn(t, u, op, nx, ny, nz)
    elif style == "dy":
        fn(t, u, op, None, nx, ny, nz)
    elif style in ("vp", "pv"):
        if routine.endswith("x" + style):
            fn(t, u, op, nx, nx, ny, nz)
        elif routine.endswith("y" + style):
            fn(t, u, op, nx, ny, ny, nz)
        else:
            fn(t, u, op, nx, ny, nz, nz)
    elif style in ("vpy", "pvy"):
        fn(t, u, op, None, nx, ny, ny, nz)


@pytest.fixture(scope="module")
def contexts(torch_cuda):
    from x3div_b200 import Context
    cache = {}

    def get(shape, prec, lengths=(2 * np.pi,) * 3):
        key = (shape, prec, lengths)
        if key not in cache:
            cache[key] = Context(*shape, lengths=lengths, precision=prec)
        return cache[key]
    yield get
    for c in cache.values():
        c.close()


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_all_routines(oracle, torch_cuda, contexts, shape, prec):
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    ctx = contexts(shape, prec)
    dt = torch.float64 if prec == "f64" else torch.float32
    u_h = seeded_field(shape, seed=sum(shape), noise=1e-2)
    u_d = to_device(u_h, dt)
    u_used = to_host(u_d).astype(np.float64)  # exactly what the kernel saw
    d = {X: ctx.dx, Y: ctx.dy, Z: ctx.dz}
    tol = 1e-12 if prec == "f64" else 1e-5
    for routine, opname, kind, direction, style in ROUTINES:
        t_d = torch.empty_like(u_d)
        call(ctx, routine, style, t_d, u_d, ctx.op(opname), shape)
        ctx.sync()
        ref = oracle.apply(kind, direction, u_used, d[direction])
        err = rel_err(to_host(t_d), ref)
        assert err < tol, (routine, opname, shape, prec, err)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("direction", [X, Y, Z])
def test_thomas_periodic_and_plain(oracle, torch_cuda, contexts, prec, direction):
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    shape = (24, 20, 16)
    ctx = contexts(shape, prec)
    dt = torch.float64 if prec == "f64" else torch.float32
    n = shape[direction]
    c = oracle.lhs("intvp", n, 0.1)
    rng = np.random.default_rng(3)
    tt_h = np.asfortranarray(rng.standard_normal(shape))
    fn = getattr(ctx, "xyz"[direction] + "thomas")
    tol = 1e-12 if prec == "f64" else 1e-5
    # periodic: ?thomas_0
    t_d = to_device(tt_h, dt)
    used = to_host(t_d).astype(np.float64)
    fn(t_d, c["f"], c["s"], c["w"], c["periodic"], c["alfa"], *shape)
    ctx.sync()
    ref = oracle.thomas_periodic(direction, used, c)
    assert rel_err(to_host(t_d), ref) < tol
    # plain: ?thomas_12
    t_d = to_device(tt_h, dt)
    fn(t_d, c["f"], c["s"], c["w"], None, 0.0, *shape)
    ctx.sync()
    ref = np.array(used, order="F", copy=True)
    oracle.lib().orc_thomas_plain(direction, oracle._p(ref), *shape, oracle._p(c["f"]),
                                  oracle._p(c["s"]), oracle._p(c["w"]))
    assert rel_err(to_host(t_d), ref) < tol


def test_operator_coefficients_match_oracle(oracle, torch_cuda, contexts):
    """x3d_operator_1d_init on the device side holds the same FP64 arrays as the oracle."""
    shape = (24, 20, 16)
    ctx = contexts(shape, "f64", (1.0, 2.0, 3.0))
    names = {"derx": ("der", 0), "deryvp": ("dervp", 1), "intzpv": ("intpv", 2), "derzz": ("der2", 2),
             "intxvp": ("intvp", 0), "derypv": ("derpv", 1)}
    for name, (kind, direction) in names.items():
        info = ctx.op(name).info()
        ref = oracle.lhs(kind, shape[direction], (1.0, 2.0, 3.0)[direction] / shape[direction])
        for key in ("f", "s", "w", "periodic"):
            np.testing.assert_allclose(info[key], ref[key], rtol=1e-15, atol=1e-15)
        for key in ("alfa", "a", "b", "c", "d"):
            assert info[key] == pytest.approx(ref[key], rel=1e-15, abs=1e-15)


def test_user_operator_roundtrip(oracle, torch_cuda, contexts):
    """x3d_op_create with arrays handed over by a host (as the Fortran
    x3d_operator_1d_init would) gives the same results as the built-in."""
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    shape = (32, 16, 8)
    ctx = contexts(shape, "f64")
    c = oracle.lhs("dervp", shape[0], ctx.dx)
    op = ctx.op_create("dervp", X, shape[0], 1, c["alfa"], c["f"], c["s"], c["w"], c["periodic"],
                       [c["a"], c["b"], c["c"], c["d"]])
    u_h = seeded_field(shape, 9)
    u = to_device(u_h)
    t1, t2 = torch.empty_like(u), torch.empty_like(u)
    ctx.derxvp(t1, u, op, *shape[:1], shape[0], *shape[1:])
    ctx.derxvp(t2, u, ctx.op("derxvp"), shape[0], shape[0], *shape[1:])
    ctx.sync()
    assert rel_err(to_host(t1), to_host(t2)) < 1e-15
    op.close()


def test_host_buffers_are_staged(oracle, torch_cuda, contexts):
    """Host (numpy) arrays through the C ABI: staged to the device and back."""
    shape = (16, 16, 16)
    ctx = contexts(shape, "f64")
    u = seeded_field(shape, 4)
    t = np.zeros_like(u, order="F")
    ctx.derz(t, u, ctx.op("derz"), *shape)
    assert rel_err(t, oracle.apply("der", Z, u, ctx.dz)) < 1e-12


def test_bad_calls_raise(torch_cuda, contexts):
    torch = torch_cuda
    from x3div_b200 import X3DError
    shape = (16, 16, 16)
    ctx = contexts(shape, "f64")
    u = torch.zeros(16, 16, 16, dtype=torch.float64, device="cuda")
    t = torch.empty_like(u)
    with pytest.raises(X3DError):   # wrong direction for the operator
        ctx.derx(t, u, ctx.op("dery"), 16, 16, 16)
    with pytest.raises(X3DError):   # non-periodic staggered sizes
        ctx.derxvp(t, u, ctx.op("derxvp"), 16, 15, 16, 16)
    with pytest.raises(X3DError):   # t aliases u (t is intent(out))
        ctx.derx(u, u, ctx.op("derx"), 16, 16, 16)
    with pytest.raises(X3DError):   # length mismatch
        ctx.derx(t, u, ctx.op("derx"), 8, 32, 16)
    ctx.sync()


@pytest.mark.parametrize("cfg", list(range(KERNEL_CONFIGS)))
@pytest.mark.parametrize("prec", ["f64", "f32"])
# (40, 60, 62): y and z lines of 4 chunks of 16 with a short last chunk,
# which the paired configurations take
@pytest.mark.parametrize("shape", [(8, 8, 8), (64, 48, 40), (100, 36, 12), (96, 20, 200), (40, 60, 62)])
def test_every_kernel_configuration(oracle, torch_cuda, contexts, cfg, prec, shape):
    """Each kernel configuration (chunked variants 0-15 and 17, one thread per
    line 16) reproduces the oracle; configurations that cannot take a shape
    fall back, and x3d_ctx_last_kernel names the one that ran."""
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    ctx = contexts(shape, prec)
    ctx.set_kernel(cfg)
    dt = torch.float64 if prec == "f64" else torch.float32
    u_d = to_device(seeded_field(shape, seed=cfg + 17, noise=1e-2), dt)
    used = to_host(u_d).astype(np.float64)
    d = {X: ctx.dx, Y: ctx.dy, Z: ctx.dz}
    tol = 1e-12 if prec == "f64" else 1e-5
    try:
        for routine, opname, kind, direction, style in ROUTINES:
            t_d = torch.empty_like(u_d)
            call(ctx, routine, style, t_d, u_d, ctx.op(opname), shape)
            ctx.sync()
            assert 0 <= ctx.last_kernel() < KERNEL_CONFIGS
            err = rel_err(to_host(t_d), oracle.apply(kind, direction, used, d[direction]))
            assert err < tol, (routine, cfg, err)
    finally:
        ctx.set_kernel(-1)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(64, 64, 64), (40, 36, 24)])
def test_grouped_batch_matches_single_calls(oracle, torch_cuda, contexts, prec, shape):
    """x3d_apply_batch: the six operator families on one input along one
    direction run as one multi-output launch and match the oracle."""
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    ctx = contexts(shape, prec)
    dt = torch.float64 if prec == "f64" else torch.float32
    u_d = to_device(seeded_field(shape, seed=5, noise=1e-2), dt)
    used = to_host(u_d).astype(np.float64)
    tol = 1e-12 if prec == "f64" else 1e-5
    kinds = ["der", "der2", "dervp", "derpv", "intvp", "intpv"]
    names = [("derx", "derxx", "derxvp", "derxpv", "intxvp", "intxpv"),
             ("dery", "deryy", "deryvp", "derypv", "intyvp", "intypv"),
             ("derz", "derzz", "derzvp", "derzpv", "intzvp", "intzpv")]
    d = (ctx.dx, ctx.dy, ctx.dz)
    for cfg in range(KERNEL_CONFIGS):
        ctx.set_kernel(cfg)
        outs = [[torch.empty_like(u_d) for _ in range(6)] for _ in range(3)]
        items = [(ctx.op(names[di][k]), u_d, outs[di][k]) for di in range(3) for k in range(6)]
        ctx.apply_batch(items)
        ctx.sync()
        for di in range(3):
            for k, kind in enumerate(kinds):
                err = rel_err(to_host(outs[di][k]), oracle.apply(kind, di, used, d[di]))
                assert err < tol, (cfg, di, kind, err)
    ctx.set_kernel(-1)
    # x3d_apply: one application, the work-list of one item
    for di in range(3):
        one = torch.empty_like(u_d)
        ctx.apply(ctx.op(names[di][2]), u_d, one)
        ctx.sync()
        assert rel_err(to_host(one), oracle.apply("dervp", di, used, d[di])) < tol, di


def test_autotune_records_choices(torch_cuda, contexts):
    shape = (64, 32, 48)
    ctx = contexts(shape, "f32")
    ctx.autotune(max_group=3)
    for direction in range(3):
        for g in (1, 2, 3):
            assert 0 <= ctx.autotune_choice(direction, g) < KERNEL_CONFIGS
    assert ctx.autotune_choice(0, 6) == -1
    ctx.set_kernel(-1)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("where", ["host_metric", "device_metric", "host_fields"])
def test_y_routines_apply_stretching_metric(oracle, torch_cuda, contexts, prec, where):
    """dery_00 / deryvp / derypv with istret /= 0 multiply the result by
    ppy(j) (ppyi(j) for deryvp) after the solve (src/x3d_derive.f90:331-337,
    src/x3d_staggered.f90:629-635, 875-881)."""
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    shape = (12, 20, 10)
    nx, ny, nz = shape
    ctx = contexts(shape, prec)
    dt = torch.float64 if prec == "f64" else torch.float32
    u_h = seeded_field(shape, seed=77, noise=1e-2)
    u_d = to_device(u_h, dt)
    u_used = to_host(u_d).astype(np.float64)
    yj = np.arange(ny) / ny
    metric = 1.0 + 0.3 * np.cos(2 * np.pi * yj) + 0.05 * yj  # > 0, not symmetric
    m_arg = torch.tensor(metric, dtype=torch.float64, device="cuda") if where == "device_metric" else metric
    tol = 1e-12 if prec == "f64" else 1e-5
    for routine, opname, kind, style in (("dery", "dery", "der", "dy"), ("dery", "deryp", "der", "dy"),
                                         ("deryvp", "deryvp", "dervp", "vpy"),
                                         ("derypv", "derypv", "derpv", "pvy")):
        op = ctx.op(opname)
        if where == "host_fields":
            u_arg = np.asfortranarray(u_used.astype(np.float64 if prec == "f64" else np.float32))
            t_arg = np.zeros_like(u_arg, order="F")
        else:
            u_arg, t_arg = u_d, torch.empty_like(u_d)
        if style == "dy":
            getattr(ctx, routine)(t_arg, u_arg, op, m_arg, nx, ny, nz)
        else:
            getattr(ctx, routine)(t_arg, u_arg, op, m_arg, nx, ny, ny, nz)
        ctx.sync()
        got = t_arg if where == "host_fields" else to_host(t_arg)
        ref = oracle.apply(kind, Y, u_used, ctx.dy) * metric[None, :, None]
        err = rel_err(np.asarray(got, dtype=np.float64), ref)
        assert err < tol, (routine, opname, prec, where, err)


# Lines longer than any staged tile holds: 4096 points (16 FP32 lines of
# 4096 need 256 KB of shared memory, above the 227 KB a CTA can have) and
# 1024-2048 points, along each direction in turn.  The library picks
# whichever kernel takes the shape; the results must not depend on it.
@pytest.mark.parametrize("shape", [(4096, 8, 8), (8, 4096, 8), (8, 8, 4096), (2048, 12, 16), (16, 1024, 24)])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_long_lines(oracle, torch_cuda, contexts, shape, prec):
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    ctx = contexts(shape, prec)
    dt = torch.float64 if prec == "f64" else torch.float32
    u_d = to_device(seeded_field(shape, seed=4096 + sum(shape), noise=1e-2), dt)
    used = to_host(u_d).astype(np.float64)
    d = {X: ctx.dx, Y: ctx.dy, Z: ctx.dz}
    tol = 1e-12 if prec == "f64" else 1e-5
    for routine, opname, kind, direction, style in ROUTINES:
        t_d = torch.empty_like(u_d)
        call(ctx, routine, style, t_d, u_d, ctx.op(opname), shape)
        ctx.sync()
        err = rel_err(to_host(t_d), oracle.apply(kind, direction, used, d[direction]))
        assert err < tol, (routine, shape, prec, err)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(64, 128, 256), (48, 64, 96)])
def test_three_ctas_per_sm_configuration(oracle, torch_cuda, contexts, prec, shape):
    """Configuration 17 (the 16-line persistent y/z kernel built for three CTAs
    per SM) runs the y and z lines it can take -- plain outputs, at most 256
    threads (16 chunks), an even chunk count -- as x3d_ctx_last_kernel shows,
    alone and as a six-operator launch, and matches the oracle."""
    torch = torch_cuda
    from x3div_b200 import to_device, to_host
    ctx = contexts(shape, prec)
    ctx.set_kernel(17)
    dt = torch.float64 if prec == "f64" else torch.float32
    u_d = to_device(seeded_field(shape, seed=1717, noise=1e-2), dt)
    used = to_host(u_d).astype(np.float64)
    d = {X: ctx.dx, Y: ctx.dy, Z: ctx.dz}
    tol = 1e-12 if prec == "f64" else 1e-5
    L = 32 if prec == "f32" else 16

    def takes(n):
        c = -(-n // L)
        return c * 16 <= 256 and (c * 16) % 32 == 0

    names = {Y: ("dery", "deryy", "deryvp", "derypv", "intyvp", "intypv"),
             Z: ("derz", "derzz", "derzvp", "derzpv", "intzvp", "intzpv")}
    kinds = ["der", "der2", "dervp", "derpv", "intvp", "intpv"]
    ran = 0
    try:
        for direction in (Y, Z):
            outs = [torch.full_like(u_d, float("nan")) for _ in range(6)]
            for k in range(6):
                ctx.apply_batch([(ctx.op(names[direction][k]), u_d, outs[k])])
                ctx.sync()
                if takes(shape[direction]):
                    assert ctx.last_kernel() == 17, (direction, k, ctx.last_kernel())
                    ran += 1
                err = rel_err(to_host(outs[k]), oracle.apply(kinds[k], direction, used, d[direction]))
                assert err < tol, (direction, kinds[k], err)
            outs = [torch.full_like(u_d, float("nan")) for _ in range(6)]
            ctx.apply_batch([(ctx.op(names[direction][k]), u_d, outs[k]) for k in range(6)])
            ctx.sync()
            if takes(shape[direction]):
                assert ctx.last_kernel() == 17
            for k in range(6):
                err = rel_err(to_host(outs[k]), oracle.apply(kinds[k], direction, used, d[direction]))
                assert err < tol, (direction, kinds[k], err)
    finally:
        ctx.set_kernel(-1)
    assert ran > 0
