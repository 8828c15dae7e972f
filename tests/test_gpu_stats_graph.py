"""GPU: reactive statistics appended to a device table from a captured CUDA
graph (lbm_reactive_stats_append_async).

Two fused fluid + A + B -> C steps (the second writing the statistics
partials) and the append are captured once and replayed three times into a
two-row table followed by a guard row: rows 0 and 1 must equal, bit for bit,
the diagnostics lbm_reactive_stats_finalize_async gives after steps 2 and 4 of
the same sequence run without a graph; the third replay must leave the guard
row untouched; the device row counter must read 3.
"""
import numpy as np
import pytest
import torch

import _util as U
import lbcube as E

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lat,real", [("D2Q9", "float"), ("D3Q19", "double")])
def test_append_from_graph_matches_finalize(engine, dev, lat, real):
    nx, ny, nz = (64, 20, 1) if lat == "D2Q9" else (16, 8, 6)
    dt = np.float32 if real == "float" else np.float64
    sl = "D2Q5" if lat == "D2Q9" else "D3Q7"
    f0 = U.random_state(lat, nx, ny, nz, dt, seed=71)
    a0 = U.random_scalar(sl, nx, ny, nz, dt, seed=72)
    b0 = U.random_scalar(sl, nx, ny, nz, dt, seed=73)
    omega, omega_c, k = 1 / 0.6, 1 / 0.8, 0.3
    pb = E.stats_partials_bytes(lat, nx, ny, nz)

    def fields():
        return ([torch.from_numpy(f0).to(dev), torch.empty(f0.shape, dtype=torch.from_numpy(f0).dtype, device=dev)],
                [torch.from_numpy(a0).to(dev), torch.empty(a0.shape, dtype=torch.from_numpy(a0).dtype, device=dev)],
                [torch.from_numpy(b0).to(dev), torch.empty(b0.shape, dtype=torch.from_numpy(b0).dtype, device=dev)])

    # plain launches: diagnostics after steps 2 and 4
    f, a, b = fields()
    part = torch.empty(pb, dtype=torch.uint8, device=dev)
    want = []
    for s in range(4):
        i, j = s % 2, (s + 1) % 2
        stats = s % 2 == 1
        E.check(E.fluid_reaction_ab_async(lat, real, "BGK", f[i], f[j], a[i], a[j], b[i], b[j], nx, ny, nz, omega,
                                          omega_c, k, part if stats else None, pb if stats else 0))
        if stats:
            d = torch.empty(8, dtype=torch.float64, device=dev)
            E.check(E.reactive_stats_finalize_async(lat, real, nx, ny, nz, k, part, pb, d))
            want.append(d)
    torch.cuda.synchronize()

    # the same two-step chunk captured once, replayed three times
    f, a, b = fields()
    table = torch.full((3, 8), -7.0, dtype=torch.float64, device=dev)  # two rows + a guard row
    row = torch.zeros(1, dtype=torch.int64, device=dev)
    s = torch.cuda.Stream(device=dev)

    def chunk():
        E.check(E.fluid_reaction_ab_async(lat, real, "BGK", f[0], f[1], a[0], a[1], b[0], b[1], nx, ny, nz, omega,
                                          omega_c, k, stream=s))
        E.check(E.fluid_reaction_ab_async(lat, real, "BGK", f[1], f[0], a[1], a[0], b[1], b[0], nx, ny, nz, omega,
                                          omega_c, k, part, pb, stream=s))
        E.check(E.reactive_stats_append_async(lat, real, nx, ny, nz, k, part, pb, table, 2, row, stream=s))

    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        chunk()
    # capturing does not run the launches: the fields are still the initial ones
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    assert int(row.item()) == 3
    assert U.same_bits(table[0].cpu().numpy(), want[0].cpu().numpy())
    assert U.same_bits(table[1].cpu().numpy(), want[1].cpu().numpy())
    assert bool((table[2] == -7.0).all()), "a row past the table was written"
    del graph
