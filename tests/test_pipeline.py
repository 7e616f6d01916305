"""HostPipeline: independent particle states streamed from pinned host memory
through several solvers on their own streams.  Each submission's result
equals a direct substep of the same state on a single solver (float atomics
in P2G order the sums differently, so positions agree to rounding)."""
import numpy as np
import pytest


def _factory(gf):
    from gpufluid_b200 import scene

    def make():
        s = gf.FlipSolver3D(32, 32, 32, transfer_mode="apic", enable_cuda_graphs=True,
                            pcg_preconditioner="tile_sgs", pcg_coarse=True)
        s.add_solid_from_sdf(scene.sdf_sphere(s.cell_centers_np(), (0.7, 0.2, 0.5), 0.12))
        s.seed_box((0.0, 0.0, 0.0), (0.4, 0.6, 1.0))
        return s
    return make


@pytest.mark.gpu
def test_pipeline_matches_direct_steps(gf):
    import torch
    from gpufluid_b200.pipeline import HostPipeline
    make = _factory(gf)
    ref = make()
    kw = dict(pressure_iters=400, pressure_solver="pcg_refined")
    states = []  # three different states: 0, 1 and 2 substeps in
    for k in range(3):
        states.append([t.detach().clone() for t in HostPipeline.state_tensors(ref)])
        ref.step(1 / 480, **kw)
    pipe = HostPipeline(make, depth=2)
    assert pipe.n == ref.n_particles and pipe.state_bytes() == ref.n_particles * 64
    ins = []
    for st in states:
        h = pipe.host_buffers()
        for a, b in zip(h, st):
            a.copy_(b)
        ins.append(h)
    outs = [pipe.host_buffers() for _ in range(6)]
    evs = [pipe.submit(ins[k % 3], outs[k], 1 / 480, **kw) for k in range(6)]
    for e in evs:
        e.synchronize()
    direct = make()
    for k in range(6):
        for d, h in zip(HostPipeline.state_tensors(direct), ins[k % 3]):
            d.copy_(h)
        direct.step(1 / 480, **kw)
        torch.cuda.synchronize()
        want = [t.cpu() for t in HostPipeline.state_tensors(direct)]
        got = outs[k]
        assert np.array_equal(got[3].numpy(), want[3].numpy())  # same storage order
        for g, w in zip(got[:3], want[:3]):
            err = np.linalg.norm(g.numpy() - w.numpy()) / max(np.linalg.norm(w.numpy()), 1e-30)
            assert err < 1e-5, (k, err)
    with pytest.raises(ValueError):
        pipe.submit(ins[0][:3], outs[0], 1 / 480, **kw)
