"""Every per-call route the library can take (afrs_ctx_set_route: the tuned
table, the generic one-launch kernel, the specialised kernels in either t <= 16
layout, the specialised kernels fused into one launch) gives the oracle's bytes
(rs/src/codec.rs:241-265 encode, :479-569 recover)."""
import numpy as np
import pytest

from oracle import oracle

torch = pytest.importorskip("torch")

ROUTES = ["AFRS_ROUTE_TABLE", "AFRS_ROUTE_GENERIC", "AFRS_ROUTE_SPECIAL", "AFRS_ROUTE_SPECIAL_SPLIT",
          "AFRS_ROUTE_FUSED", "AFRS_ROUTE_FEW"]


def test_set_route_argument_checks(afrs):
    lib, E = afrs.lib(), afrs._lib.AFRS_EINVAL
    assert lib.afrs_ctx_set_route(None, 0) == E


@pytest.mark.gpu
def test_set_route_rejects_unknown_values(afrs):
    ctx = afrs.Context(0)
    with pytest.raises(afrs.AfrsError):
        ctx.set_route(6)
    with pytest.raises(afrs.AfrsError):
        ctx.set_route(-1)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("route", ROUTES)
@pytest.mark.parametrize("n,t,L", [(64, 4, 3000), (64, 16, 1029), (256, 8, 2048), (128, 64, 777), (32, 16, 64),
                                   (16, 4, 5000), (256, 128, 4096)])
def test_encode_routes_match_oracle(afrs, route, n, t, L):
    msg = oracle.random_bytes((n - t) * L, n + t + L)
    p0 = oracle.random_bytes(t * L, 3)
    ref = p0.copy()
    oracle.encode_systematic_sharded(n, t, msg, ref, L)
    ctx = afrs.Context(0)
    ctx.set_route(getattr(afrs._lib, route))
    d = torch.from_numpy(p0.copy()).cuda()
    afrs.Codec(n, t, context=ctx).encode_systematic_sharded(torch.from_numpy(msg).cuda(), d, None, L)
    assert (d.cpu().numpy() == ref).all()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("route", ROUTES)
@pytest.mark.parametrize("n,t,L", [(64, 32, 1024), (16, 8, 3000), (256, 128, 2048), (32, 4, 777), (8, 2, 100)])
def test_recover_routes_match_oracle(afrs, route, n, t, L):
    msg = oracle.random_bytes((n - t) * L, n * 3 + L)
    par = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, par, L)
    cw = np.concatenate([par, msg])
    pos = sorted(np.random.default_rng(n + t).choice(n, t, replace=False).tolist())
    rx = cw.copy()
    for p in pos:
        rx[p * L:(p + 1) * L] = 0
    ctx = afrs.Context(0)
    ctx.set_route(getattr(afrs._lib, route))
    d = torch.from_numpy(rx).cuda()
    assert afrs.Codec(n, t, context=ctx).recover_erasure_shards(d, None, L, pos)
    assert (d.cpu().numpy() == cw).all()
    ctx.close()


# Shapes of the one-launch form: encodes with t = 32, 64 (every chunk count),
# recovers with n = 32 .. 128; shard lengths with partial last slices, one
# slice, several slices.
FUSED_LENGTHS = [64, 777, 1024, 3000, 4096 + 37]


@pytest.mark.gpu
@pytest.mark.parametrize("n,t", [(64, 32), (128, 32), (128, 64), (256, 32), (256, 64)])
@pytest.mark.parametrize("L", FUSED_LENGTHS)
def test_fused_encode_matches_oracle(afrs, n, t, L):
    msg = oracle.random_bytes((n - t) * L, 7 * n + t + L)
    p0 = oracle.random_bytes(t * L, L)
    ref_acc = p0.copy()
    oracle.encode_systematic_sharded(n, t, msg, ref_acc, L)
    ref = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, ref, L)
    ctx = afrs.Context(0)
    ctx.set_route(afrs._lib.AFRS_ROUTE_FUSED)
    codec = afrs.Codec(n, t, context=ctx)
    d_msg = torch.from_numpy(msg).cuda()
    d = torch.from_numpy(p0.copy()).cuda()
    codec.encode_systematic_sharded(d_msg, d, None, L)  # XOR-accumulates into the parity
    assert (d.cpu().numpy() == ref_acc).all()
    d.fill_(0x5A)
    codec.encode_parity(d_msg, d, L)  # parity overwritten
    assert (d.cpu().numpy() == ref).all()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [32, 64, 128])
@pytest.mark.parametrize("L", FUSED_LENGTHS)
@pytest.mark.parametrize("pattern", ["one", "half", "all_t_random", "run"])
def test_fused_recover_matches_oracle(afrs, n, L, pattern):
    t = n // 2
    msg = oracle.random_bytes((n - t) * L, 11 * n + L)
    par = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, par, L)
    cw = np.concatenate([par, msg])
    rng = np.random.default_rng(n + L)
    pos = {"one": [n - 1], "half": rng.choice(n, t // 2, replace=False).tolist(),
           "all_t_random": rng.choice(n, t, replace=False).tolist(),
           "run": list(range(5, 5 + t))}[pattern]
    rx = cw.copy()
    for p in pos:
        rx[p * L:(p + 1) * L] = 0
    ctx = afrs.Context(0)
    ctx.set_route(afrs._lib.AFRS_ROUTE_FUSED)
    d = torch.from_numpy(rx).cuda()
    assert afrs.Codec(n, t, context=ctx).recover_erasure_shards(d, None, L, sorted(pos))
    assert (d.cpu().numpy() == cw).all()
    ctx.close()
