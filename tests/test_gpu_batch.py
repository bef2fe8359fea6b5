"""Box batches: one persistent launch sweeping uneven boxes, checked against
the oracle for every operator family and direction, plain and graph-replayed."""
import numpy as np
import pytest

from conftest import rel_err, seeded_field

pytestmark = pytest.mark.gpu

KINDS = ["der", "der2", "dervp", "derpv", "intvp", "intpv"]
# (18, 12, 10): in FP32 its rows are 72 bytes, not a multiple of 16, so the box
# runs through the fallback launches; in FP64 (144-byte rows) it joins the batch
BOXES = [(16, 16, 16), (24, 20, 12), (32, 8, 16), (64, 40, 24), (18, 12, 10), (96, 36, 20)]


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_batch_sweep_matches_oracle(oracle, torch_cuda, prec):
    torch = torch_cuda
    from x3div_b200 import Batch, to_device, to_host
    dt = torch.float32 if prec == "f32" else torch.float64
    tol = 1e-5 if prec == "f32" else 1e-12
    nf = 2
    fields, outs, used = [], [], []
    for i, b in enumerate(BOXES):
        fs = [to_device(seeded_field(b, 100 * i + f, noise=1e-2), dt) for f in range(nf)]
        fields.append(fs)
        used.append([to_host(a).astype(np.float64) for a in fs])
        outs.append([[[torch.full_like(fs[0], np.nan) for _ in range(6)] for _ in range(3)] for _ in range(nf)])
    batch = Batch(BOXES, precision=prec)
    batch.bind_sweep(fields, outs)
    info = batch.info()
    assert info["fallback_jobs"] == (3 * nf if prec == "f32" else 0)  # only the odd box
    assert info["points"] == 18 * nf * sum(b[0] * b[1] * b[2] for b in BOXES)

    def check():
        for i, b in enumerate(BOXES):
            d = [2 * np.pi / n for n in b]
            for f in range(nf):
                for di in range(3):
                    for k, kind in enumerate(KINDS):
                        ref = oracle.apply(kind, di, used[i][f], d[di])
                        err = rel_err(to_host(outs[i][f][di][k]), ref)
                        assert err < tol, (b, f, di, kind, err)

    batch.run()
    batch.sync()
    check()
    for i in range(len(BOXES)):
        for f in range(nf):
            for di in range(3):
                for k in range(6):
                    outs[i][f][di][k].fill_(np.nan)
    batch.capture()
    batch.replay()
    batch.replay()
    batch.sync()
    check()
    batch.close()


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_batch_autotune_keeps_results(oracle, torch_cuda, prec):
    """x3d_batch_autotune picks a chunk length and tile width per box shape
    and direction (x3d_batch_choice reports them); the re-planned persistent
    launch still matches the oracle, plainly and from its CUDA graph."""
    torch = torch_cuda
    from x3div_b200 import Batch, to_device, to_host
    dt = torch.float32 if prec == "f32" else torch.float64
    tol = 1e-5 if prec == "f32" else 1e-12
    boxes = [(16, 16, 16), (24, 20, 12), (64, 40, 24), (16, 16, 16), (96, 36, 20)]
    fields, outs, used = [], [], []
    for i, b in enumerate(boxes):
        fs = [to_device(seeded_field(b, 300 + 10 * i + f, noise=1e-2), dt) for f in range(2)]
        fields.append(fs)
        used.append([to_host(a).astype(np.float64) for a in fs])
        outs.append([[[torch.full_like(fs[0], np.nan) for _ in range(6)] for _ in range(3)] for _ in range(2)])
    batch = Batch(boxes, precision=prec)
    batch.bind_sweep(fields, outs)
    batch.autotune()
    long_chunk, short_chunk = (32, 16) if prec == "f32" else (16, 8)
    for i in range(len(boxes)):
        for d in range(3):
            chunk, lines = batch.choice(i, d)
            assert chunk in (long_chunk, short_chunk) and lines > 0, (boxes[i], d, chunk, lines)
    assert batch.choice(0, 1) == batch.choice(3, 1)  # one choice per shape

    def check():
        for i, b in enumerate(boxes):
            h = [2 * np.pi / n for n in b]
            for f in range(2):
                for d in range(3):
                    for k, kind in enumerate(KINDS):
                        err = rel_err(to_host(outs[i][f][d][k]), oracle.apply(kind, d, used[i][f], h[d]))
                        assert err < tol, (b, f, d, kind, err)

    for per_box in outs:
        for per_f in per_box:
            for per_d in per_f:
                for o in per_d:
                    o.fill_(np.nan)
    batch.run()
    batch.sync()
    check()
    batch.capture()
    batch.replay()
    batch.sync()
    check()
    batch.close()
