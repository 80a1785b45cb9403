"""View sharding of one object across ranks (ct_forward_projection_b200.shard),
host logic on CPU: two and three `gloo` ranks (7 views in slabs of 4 + 3 and
3 + 2 + 2), each with a stand-in projector that computes its view range with
the FP64 oracle (test infrastructure), must give
the single-process projection (all-gather) and gradient (all-reduce)."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from ct_forward_projection_b200.shard import ViewShardedProjector, view_range
from tests.conftest import random_volumes, small_geometry, spectral_setup


@pytest.mark.parametrize("P,world", [(1, 1), (7, 2), (8, 2), (5, 3), (360, 8), (3, 4)])
def test_view_ranges_cover_each_view_once(P, world):
    seen = []
    for r in range(world):
        first, n = view_range(P, r, world)
        assert n >= 0
        seen.extend(range(first, first + n))
    assert seen == list(range(P))
    sizes = [view_range(P, r, world)[1] for r in range(world)]
    assert max(sizes) - min(sizes) <= 1


def test_view_range_rejects_bad_rank():
    with pytest.raises(ValueError):
        view_range(4, 2, 2)


GEOM = dict(n=(10, 9, 8), views=7, U=9, V=6)


class OracleProjector:
    """Stand-in with the Projector interface the sharder uses, on CPU tensors:
    forward/backward over a view range through the FP64 oracle."""

    def __init__(self, d, M, S, mu, G, D):
        from oracle import oracle as O
        self.O, self.d, self.M, self.mu = O, d, M, mu
        self.W = O.energy_weights(d, S, G, 2, D, 1000.0)
        self.shape_proj = (d["projNum"], d["dNumV"], d["dNumU"])

    def _ids(self, views):
        npix = self.d["dNumU"] * self.d["dNumV"]
        return np.arange(views[0] * npix, (views[0] + views[1]) * npix, dtype=np.int64)

    def forward(self, volumes, want_L=False, views=None):
        n = views[1]
        _, V, U = self.shape_proj
        r = self.O.forward(self.d, [v.numpy() for v in volumes], self.mu, self.W, self.O.TRILINEAR,
                           self._ids(views))
        out = {"I": torch.from_numpy(r["I"].reshape(n, V, U)), "IAbsorb": torch.from_numpy(r["IAbsorb"].reshape(n, V, U))}
        if want_L:
            out["L"] = torch.from_numpy(r["L"].reshape(n, V, U, self.M))
        return out

    def backward(self, L, gI=None, gIAbsorb=None, grads=None, views=None):
        g = self.O.backward(self.d, self.mu, self.W, L.numpy().reshape(-1, self.M),
                            None if gI is None else gI.numpy().ravel(), None, self.O.TRILINEAR, self._ids(views))
        if grads is None:
            return [torch.from_numpy(x) for x in g]
        for a, b in zip(grads, g):
            a += torch.from_numpy(b)
        return grads


def _setup():
    d = small_geometry(n=GEOM["n"], views=GEOM["views"], U=GEOM["U"], V=GEOM["V"])
    M = 2
    vols = [torch.from_numpy(v) for v in random_volumes(d, M, 21)]
    S, mu, G, D = spectral_setup(d, M, 5, 3)
    return d, M, vols, S, mu, G, D


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d, M, vols, S, mu, G, D = _setup()
        sp = ViewShardedProjector(OracleProjector(d, M, S, mu, G, D))
        f = sp.forward(vols, want_L=True, gather=True)
        gI = torch.from_numpy(np.linspace(-1.0, 1.0, f["I"].numel()).reshape(f["I"].shape))
        gI = gI * 1e-3 + 1e-4 * sp.views[0]
        grads = sp.backward(f["L"], gI=gI)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), I=f["I_full"].numpy(), A=f["IAbsorb_full"].numpy(),
                 g0=grads[0].numpy(), g1=grads[1].numpy(), v0=sp.views[0], n=sp.views[1])
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("world", [2, 3])
def test_view_sharded_forward_and_adjoint_match_one_process(world):
    with tempfile.TemporaryDirectory() as td:
        mp.start_processes(_rank_main, args=(world, _free_port(), td), nprocs=world, join=True, start_method="spawn")
        outs = [np.load(os.path.join(td, f"r{r}.npz")) for r in range(world)]
    d, M, vols, S, mu, G, D = _setup()
    pr = OracleProjector(d, M, S, mu, G, D)
    P = d["projNum"]
    full = pr.forward(vols, want_L=True, views=(0, P))
    # the gradient each rank fed in, assembled over the full view range
    gI = []
    for o in outs:
        n = int(o["n"])
        gI.append(np.linspace(-1.0, 1.0, n * d["dNumV"] * d["dNumU"]).reshape(n, d["dNumV"], d["dNumU"]) * 1e-3
                  + 1e-4 * int(o["v0"]))
    ref = pr.backward(full["L"], gI=torch.from_numpy(np.concatenate(gI)), views=(0, P))
    for o in outs:
        np.testing.assert_array_equal(o["I"], full["I"].numpy())
        np.testing.assert_array_equal(o["A"], full["IAbsorb"].numpy())
        for m in range(M):
            np.testing.assert_allclose(o[f"g{m}"], ref[m].numpy(), rtol=1e-12, atol=1e-15)
