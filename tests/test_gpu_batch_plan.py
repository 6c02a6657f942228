"""Prepared batches (afrs_batch_plan_*): a plan built once runs its jobs on
every launch, bit-exact with the oracle (rs/src/codec.rs:241-265 encode,
:479-569 recover), also when its launch is captured into a CUDA graph and
the graph is replayed on fresh contents of the same buffers."""
import numpy as np
import pytest

from oracle import oracle

torch = pytest.importorskip("torch")


def test_plan_argument_checks(afrs):
    import ctypes

    lib, E = afrs.lib(), afrs._lib.AFRS_EINVAL
    h = ctypes.c_void_p()
    assert lib.afrs_batch_plan_create(None, None, 0, ctypes.byref(h)) == E
    assert lib.afrs_batch_plan_launch(None, None) == E
    lib.afrs_batch_plan_destroy(None)


def _jobs(afrs, seed):
    """Small mixed jobs (the generic persistent kernel) plus one shape group
    large enough for the grouped kernels (32 recovers, n = 128, 2 KiB)."""
    rng = np.random.default_rng(seed)
    jobs, refs, inputs = [], [], []
    shapes = [(int(rng.choice([32, 64])), 8, int(rng.choice([64, 320, 1024]))) for _ in range(40)]
    shapes += [(128, 64, 2048)] * 32
    for i, (n, t, L) in enumerate(shapes):
        msg = oracle.random_bytes((n - t) * L, seed * 1000 + i)
        par = np.zeros(t * L, np.uint8)
        oracle.encode_systematic_sharded(n, t, msg, par, L)
        if i < 40 and i % 2 == 0:
            jobs.append(afrs.Job.encode(n, t, torch.from_numpy(msg).cuda(),
                                        torch.zeros(t * L, dtype=torch.uint8, device="cuda"), L))
            refs.append(par)
            inputs.append(msg)
        else:
            cw = np.concatenate([par, msg])
            e = int(rng.integers(1, t + 1))
            pos = sorted(rng.choice(n, e, replace=False).tolist())
            rx = cw.copy()
            for p in pos:
                rx[p * L:(p + 1) * L] = 0
            jobs.append(afrs.Job.recover(n, t, torch.from_numpy(rx).cuda(), L, pos))
            refs.append(cw)
            inputs.append(rx)
    return jobs, refs, inputs


def _reset(jobs, inputs):
    for j, x in zip(jobs, inputs):
        if j.op == 0:
            j.dst.zero_()
        else:
            j.dst.copy_(torch.from_numpy(x))


@pytest.mark.gpu
def test_plan_launches_match_oracle(afrs):
    jobs, refs, inputs = _jobs(afrs, 3)
    plan = afrs.BatchPlan(jobs)
    assert plan.statuses == [0 if j.op == 0 else 1 for j in jobs]
    for _ in range(2):
        _reset(jobs, inputs)
        plan.launch()
        torch.cuda.synchronize()
        for j, r in zip(jobs, refs):
            assert (j.dst.cpu().numpy() == r).all()
    plan.close()


@pytest.mark.gpu
def test_plan_launch_in_a_cuda_graph(afrs):
    jobs, refs, inputs = _jobs(afrs, 4)
    plan = afrs.BatchPlan(jobs)
    plan.launch()  # first launch outside the capture (kernel set-up)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with torch.cuda.graph(g, stream=s):
        plan.launch()
    for _ in range(2):
        _reset(jobs, inputs)
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        for j, r in zip(jobs, refs):
            assert (j.dst.cpu().numpy() == r).all()
    del g
    plan.close()


@pytest.mark.gpu
def test_grouped_scratch_rounds(afrs):
    """A batch whose grouped jobs need more scratch than one round holds
    (1 GiB): nine n = 256 recovers with 512 KiB shards need 268 MB each, so
    they run in three rounds that reuse the scratch, next to nine encodes of
    the same shape.  Each recover must give back its original codeword and
    each encode the per-call encoder's parity (itself checked against the
    oracle by the parity tests), through afrs_batch_dev and through a plan
    launched twice."""
    n, t, L, K = 256, 128, 512 << 10, 9
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    codec = afrs.Codec(n, t)
    rng = np.random.default_rng(17)
    cws, rxs, msgs, pars, patterns = [], [], [], [], []
    for i in range(K):
        cw = torch.empty(n * L, dtype=torch.uint8, device="cuda")
        cw[t * L:] = torch.randint(0, 256, ((n - t) * L,), dtype=torch.uint8, device="cuda", generator=g)
        codec.encode_parity(cw[t * L:], cw[:t * L], L)
        pos = sorted(rng.choice(n, t, replace=False).tolist())
        rx = cw.clone()
        for p in pos:
            rx[p * L:(p + 1) * L].zero_()
        cws.append(cw)
        rxs.append(rx)
        patterns.append(pos)
        msgs.append(cw[t * L:].clone())
        pars.append(torch.full((t * L,), 0x5A, dtype=torch.uint8, device="cuda"))

    def jobs():
        out = [afrs.Job.recover(n, t, rxs[i], L, patterns[i]) for i in range(K)]
        out += [afrs.Job.encode(n, t, msgs[i], pars[i], L) for i in range(K)]
        return out

    def check():
        torch.cuda.synchronize()
        for i in range(K):
            assert torch.equal(rxs[i], cws[i]), f"recover {i}"
            assert torch.equal(pars[i], cws[i][:t * L]), f"encode {i}"

    def reset():
        for i in range(K):
            for p in patterns[i]:
                rxs[i][p * L:(p + 1) * L].zero_()
            pars[i].fill_(0x5A)

    statuses = afrs.run_batch(jobs())
    assert statuses == [1] * K + [0] * K
    check()
    js = jobs()
    reset()
    plan = afrs.BatchPlan(js)
    for _ in range(2):
        plan.launch()
        check()
        reset()
    plan.close()
