"""og_gb_energy_noalloc: the GB solvation energy for callers that cannot
allocate device memory when they need it (their GPU memory is reserved up
front by another allocator, or their loop forbids allocation after start-up).

The entry point keeps its scratch in a fixed array inside the library, so
this test hands it only device buffers the test owns (torch tensors).  It
makes the set-up call first (n_atoms = 0, every pointer NULL: loads the
kernels and the array on the device), then checks two calls in a row -- on
two different conformations, so a second call cannot pass on what the first
left in the shared scratch -- against the engine's own FP64 energy path
(og_compute_energies) and against the FP64 CPU oracle, within the 1e-6
relative tolerance of the other energy tests, and checks that the device's
free memory is the same before and after a call.  Collected last so that a
run stopping at its first failure has already run every other test.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import Orc

pytestmark = pytest.mark.gpu

TRP = "NLYIQWLKDGGPSSGRPPPS"


def _dev(t):
    return t.data_ptr()


def test_gb_energy_noalloc_matches_engine(origami):
    import torch

    lib = origami.lib()
    chain = origami.Chain.build(TRP, math.radians(-57.0), math.radians(-47.0), math.pi)
    topo = chain.topology()
    x1 = chain.positions
    x2 = x1 + np.random.default_rng(7).normal(scale=0.05, size=x1.shape)
    dev = torch.device("cuda:0")
    q = torch.tensor(topo.charge, dtype=torch.float64, device=dev)
    rho = torch.tensor(topo.gb_rho, dtype=torch.float64, device=dev)
    scale = torch.tensor(topo.gb_scale, dtype=torch.float64, device=dev)
    out = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    n = chain.n_atoms
    assert lib.og_gb_energy_noalloc(None, None, None, None, 0, 20.0, None, stream) == 0, lib.og_last_error()

    for x in (x1, x2):
        eng = origami.Engine(origami.Params())
        eng.add_system(chain, x, 310.0)
        eng.finalize()
        ref = eng.energies(0)
        eng.close()

        orc = Orc(chain).energy_terms(x, nb=10.0, born=20.0)

        xyz = torch.tensor(x.reshape(-1), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        st = lib.og_gb_energy_noalloc(_dev(xyz), _dev(q), _dev(rho), _dev(scale), n, 20.0, _dev(out), stream)
        assert st == 0, lib.og_last_error()
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info(dev)[0] == free_before  # the call took no device memory
        gb, self_e, pair = out.tolist()
        for got, want, oracle_want in ((gb, ref["gb"], orc["gb"]), (self_e, ref["gb_self"], orc["gb_self"]),
                                       (pair, ref["gb_pair"], orc["gb_pair"])):
            assert abs(got - want) <= 1e-6 * max(abs(want), 1.0), (got, want)
            assert abs(got - oracle_want) <= 1e-6 * max(abs(oracle_want), 1.0), (got, oracle_want)


def test_gb_energy_noalloc_rejects_oversized_systems(origami):
    import torch

    lib = origami.lib()
    dev = torch.device("cuda:0")
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    p = buf.data_ptr()
    limit = 16384  # OG_NOALLOC_MAX_ATOMS
    assert lib.og_gb_energy_noalloc(p, p, p, p, limit + 1, 20.0, p, None) == 1  # OG_E_BADARG
    assert b"n_atoms" in lib.og_last_error()
    assert lib.og_gb_energy_noalloc(p, p, p, p, 0, 20.0, p, None) == 1
