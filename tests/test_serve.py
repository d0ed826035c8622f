"""Replica server (continuous batching): admission by memory budget, and each
replica's result identical alone and in the mix (mixed precision: bit-exact,
the force sums are integer sums)."""
import numpy as np
import pytest

from thrid_b200 import abi
from thrid_b200 import systems as S


def _replicas():
    return [S.small_box("water", nside=4, spacing=3.1, precision=abi.PREC_MIXED, seed=3),
            S.small_box("propanol", nside=3, spacing=5.6, precision=abi.PREC_MIXED, seed=5),
            S.small_box("butane", nside=4, spacing=5.4, precision=abi.PREC_MIXED, nfft=24, order=5, seed=9)]


def test_estimate_bytes_grows_with_size():
    from thrid_b200.serve import estimate_bytes
    a = estimate_bytes(S.small_box("propanol", nside=3, spacing=5.6))
    b = estimate_bytes(S.small_box("propanol", nside=5, spacing=5.6))
    assert 0 < a < b


@pytest.mark.gpu
def test_results_identical_alone_and_in_the_mix():
    from thrid_b200.serve import ReplicaServer
    reps = _replicas()
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    alone = []
    srv = ReplicaServer(max_slots=1)
    for s in reps:
        rid = srv.submit(s, md, kind=0, nsteps=40)
        alone.append(srv.result(rid))
    srv.close()
    srv = ReplicaServer(max_slots=3)
    ids = [srv.submit(s, md, kind=0, nsteps=40) for s in reps]
    mixed = [srv.result(r) for r in ids]
    srv.close()
    # the replicas overlapped in time
    starts = [m[5][1] for m in mixed]
    dones = [m[5][2] for m in mixed]
    assert max(starts) < min(dones)
    for a, m in zip(alone, mixed):
        assert np.array_equal(a[0], m[0]) and np.array_equal(a[1], m[1])
        assert a[3]["pot_tot"] == m[3]["pot_tot"]


@pytest.mark.gpu
def test_admission_respects_the_memory_budget():
    from thrid_b200.serve import ReplicaServer, estimate_bytes
    reps = _replicas()[:2]
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    budget = max(estimate_bytes(s) for s in reps) + 1      # room for one replica at a time
    srv = ReplicaServer(max_slots=2, hbm_budget_bytes=budget)
    ids = [srv.submit(s, md, kind=0, nsteps=30) for s in reps]
    r = [srv.result(i) for i in ids]
    srv.close()
    assert r[1][5][1] >= r[0][5][2]                         # second admitted after the first finished


@pytest.mark.gpu
def test_heat_flux_replica_through_the_server():
    from thrid_b200.serve import ReplicaServer
    s = S.slab_box(nxy_w=6, nlay_w=6, nwater=216, nxy_p=3, nlay_p=1, lxy=18.6, rcut=7.0, nfft=(16, 16, 64),
                   vacuum=8.0, hf_width=5.0, precision=abi.PREC_MIXED)
    hf = dict(s.regions["hf"])
    hf["heatfinterval"] = 2
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    srv = ReplicaServer(max_slots=2)
    rid = srv.submit(s, md, kind=3, nsteps=6, hf=hf)
    x, v, box, e, rec, t = srv.result(rid)
    srv.close()
    assert rec.shape == (3, len(hf["regions"]), abi.HF_NCOL)
    assert np.isfinite(rec).all() and np.isfinite(x).all()
