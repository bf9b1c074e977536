"""GPU: the Hessian producer (stg_fem_newton_system) against the CPU assembly of the
synthetic scenes (stgipc/scenes._assemble): same converted BCOO pattern, blocks and
gradient to FP64 rounding (summation order and eigen-solver differ), barriers active on
both planes, and the solve of the GPU-built system matching the CPU-built one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,seed", [(6, 2400), (10, 2401)])
def test_newton_system_matches_cpu_assembly(dev, n, seed):
    from oracle import oracle as orc
    from stgipc import fem, scenes
    st = scenes.make_heterogeneous_cube(n=n, seed=seed, state_only=True)
    cpu = scenes._assemble(**st)
    rows, cols, blocks, b = fem.newton_system(st["pos_rest"], st["pos"], st["vel"], st["tets"], st["E"], st["nu"],
                                              st["rho"], st["dt"], st["barriers"], device=dev)
    assert rows.numel() == 10 * st["tets"].shape[0] + cpu.num_verts
    rg, cg, bg = orc.convert(rows.cpu().numpy(), cols.cpu().numpy(), blocks.cpu().numpy())
    rc, cc, bc = orc.convert(cpu.rows, cpu.cols, cpu.blocks)
    np.testing.assert_array_equal(rg, rc)
    np.testing.assert_array_equal(cg, cc)
    scale = np.abs(bc).max()
    assert np.abs(bg - bc).max() <= 1e-10 * scale
    bb = b.cpu().numpy()
    assert np.abs(bb - cpu.b).max() <= 1e-10 * np.abs(cpu.b).max()
    # both barrier planes are active in this state
    y = st["pos"][:, 1]
    assert (y < st["barriers"][0][2]).any() and ((-y + st["barriers"][1][1]) < st["barriers"][1][2]).any()


def test_gpu_built_system_solves_like_cpu_built(dev):
    import torch
    from stgipc import PCGSolverConfig, Solver, fem, scenes
    st = scenes.make_heterogeneous_cube(n=12, seed=2402, state_only=True)
    cpu = scenes._assemble(**st)
    rows, cols, blocks, b = fem.newton_system(st["pos_rest"], st["pos"], st["vel"], st["tets"], st["E"], st["nu"],
                                              st["rho"], st["dt"], st["barriers"], device=dev)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    out = []
    for R, C, B, bb in ((rows, cols, blocks.reshape(-1), b), (t(cpu.rows), t(cpu.cols), t(cpu.blocks.reshape(-1)),
                                                               t(cpu.b))):
        s = Solver(PCGSolverConfig(precision="fp64", stop_rule="relative_residual", global_tol_rate=1e-6))
        s.mas_init(cpu.num_verts, cpu.neighbor_start, cpu.neighbor_num, cpu.neighbor_list, *cpu.slot_maps(16))
        x = torch.zeros_like(bb)
        stt = s.solve_linear_system(R, C, B, bb, x)
        out.append((stt["iterations"], x.cpu().numpy()))
    assert abs(out[0][0] - out[1][0]) <= 1
    assert np.linalg.norm(out[0][1] - out[1][1]) <= 1e-6 * np.linalg.norm(out[1][1])
