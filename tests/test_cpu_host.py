"""CPU-only checks of the product's host side: the C-ABI library loads and
exports every symbol declared in include/krans_cuda.h, the Python mirror maps
the reference's option names and defaults, and the generators produce the
exact kernels they claim. No GPU is touched."""
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "krans_cuda.h")).read()
    return set(re.findall(r"^(?:int|const char \*)\s*(krans_[a-z0-9_]+)\(", txt, flags=re.M))


def test_library_exports_every_declared_symbol():
    from krans_b200 import _capi, build
    build.build()
    have = _capi.exported_symbols()
    want = declared_symbols()
    assert want, "no declarations parsed"
    assert want <= set(_capi.SIGNATURES), want - set(_capi.SIGNATURES)
    assert want <= have, want - have
    lib = _capi.load()
    assert b"sm_100a" in lib.krans_version()


def test_context_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import krans_b200 as kb
    with pytest.raises(kb.KransError):
        kb.Context(0)


def test_option_defaults_mirror_reference():
    # CyclicLanczosSolver.hpp:84-146, LOBPCGSolver.hpp:71-115
    import krans_b200 as kb
    o = kb.CyclicLanczosOptions()
    assert (o.k, o.ncv, o.max_restarts, o.tol_abs, o.tol_rel) == (1, 48, 80, 1e-12, 1e-10)
    assert o.reorth == kb.ReorthMode.Double and o.use_harmonic and o.target_tau == 0.0
    assert (o.cg_maxit, o.cg_rel_tol, o.cg_breakdown_tol, o.projector_passes) == (80, 1e-10, 1e-30, 1)
    assert (o.grad_max_iters, o.frob_samples, o.prescreen_factor, o.stagnation_restarts) == (3000, 4, 0.8, 30)
    c = o.to_c()
    assert c.ncv == 48 and c.reorth == 2 and c.stagnation_restarts == 30 and c.precision == 0
    # engine knob: a mixed solve that stalls in its polish continues in FP64 unless told otherwise
    assert o.mixed_fallback and c.mixed_fallback == 1
    assert kb.CyclicLanczosOptions(mixed_fallback=False).to_c().mixed_fallback == 0
    L = kb.LOBPCGOptions()
    assert (L.nev, L.block_size, L.max_iters, L.restart, L.gs_tol) == (1, 0, 1000, 0.9, 1e-14)
    assert L.soft_locking and L.gs_reorth and L.frob_samples == 4 and L.nullity_known == -1
    assert L.to_c().max_iters == 1000


def test_generators_exact_kernels():
    from krans_b200 import generators as G
    for inst in [G.shift_operator(300, 4, 0.7), G.difference_operator(50),
                 G.graph_incidence(2000, 5, 6.0, seed=3), G.planted_kernel(1500, 1000, 6, seed=2)]:
        K = inst.kernel
        assert K.shape[0] == inst.k
        assert np.allclose(K @ K.T, np.eye(inst.k), atol=1e-12)
        assert np.linalg.norm(inst.A @ K.T) <= 1e-12 * max(1.0, sp.linalg.norm(inst.A))
    gi = G.graph_incidence(2000, 5, 6.0, seed=3)
    assert gi.A.shape == (6000, 2000) and np.all(np.diff(gi.A.indptr) == 2)
    pk = G.planted_kernel(1500, 1000, 6, seed=2)
    B = pk.A[:, :1000]
    assert np.all(np.diff(B.tocsc().indptr) > 0)  # every column of B nonempty
    bi = G.batch_instances(6, seed=1)
    assert [i.name for i in bi] == ["shift", "incidence"] * 3


def test_replicas_gloo_two_ranks(tmp_path):
    """The multi-GPU form is replicas only (independent requests, no data-path
    collective); the host reduction of per-rank times/counts is a max and a
    sum. Checked with two gloo ranks on the CPU."""
    import torch.multiprocessing as mp
    mp.start_processes(_replica_worker, args=(2, str(tmp_path)), nprocs=2, start_method="spawn")
    vals = [float(open(tmp_path / f"r{r}").read()) for r in range(2)]
    assert vals == [2.0, 2.0]


def _replica_worker(rank, world, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT="29533")
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = torch.tensor([1.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    open(os.path.join(out, f"r{rank}"), "w").write(str(float(t)))
    dist.destroy_process_group()


def test_abi_struct_sizes_match_the_library():
    # the ctypes mirrors of the C ABI structs (krans_b200/_capi.py) against
    # sizeof() as the library was compiled (krans_abi_sizes; no GPU needed)
    import ctypes as C
    from krans_b200 import _capi as K
    lib = K.load()
    out = (C.c_int64 * 9)()
    assert lib.krans_abi_sizes(out, 9) == 9
    mine = [K.CyclicOpts, K.CyclicResultC, K.LobpcgOpts, K.LobpcgResultC, K.Request, K.RequestResult,
            K.ServerOpts, K.SpmvTuning, K.BatchTuning]
    assert [C.sizeof(t) for t in mine] == list(out)
