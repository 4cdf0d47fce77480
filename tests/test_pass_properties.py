"""Properties of the whole flux pass (the oracle restatement, pinned bit for
bit against the reference's pass) on the committed meshes: total mass is
conserved to round-off in a closed box, and so is total energy unless get_W
floors a cell's pressure at 1e-30 (it then rewrites that cell's energy, as the
reference does: src/riemann/ExactRiemannSolver.cpp:740-766); a uniform state
at rest stays as it is (each closed cell's face area vectors sum to zero)."""
import numpy as np
import pytest

from golden_util import load_case
from oracle.oracle import Params


@pytest.mark.parametrize("name", ["sod2d_exact", "sod2d_hllc", "sedov3d_hllc",
                                  "random3d_exact", "random2d_periodic_exact"])
def test_mass_and_energy_are_conserved(oracle, name):
    mesh, meta, _ = load_case(name)
    D = mesh.dim
    p = Params(solver=meta["solver"], gamma=meta["gamma"])
    W0 = meta["W0"]
    V = mesh.cell_volume
    m0 = (W0[:, 0] * V).sum()
    e0 = ((W0[:, D + 1] / (meta["gamma"] - 1.0)
           + 0.5 * W0[:, 0] * (W0[:, 1:D + 1] ** 2).sum(1)) * V).sum()
    floored = False
    for k in range(1, meta["nsteps"] + 1):
        out = oracle.run(mesh, p, meta["dt"], k, W0)
        assert out["status"] == 0
        floored |= bool(np.any(out["W"][:, D + 1] <= 1e-30))
    Q = out["Q"]
    assert abs(Q[:, 0].sum() - m0) <= 1e-13 * m0
    if name == "random2d_periodic_exact":
        assert floored      # the supersonic random field empties a cell
    else:
        assert not floored
        assert abs(Q[:, D + 1].sum() - e0) <= 1e-12 * e0


@pytest.mark.parametrize("name", ["sod2d_exact", "sedov3d_hllc", "random2d_periodic_exact"])
def test_uniform_state_at_rest_stays(oracle, name):
    mesh, meta, _ = load_case(name)
    D = mesh.dim
    W0 = np.zeros((mesh.n_cells, D + 2))
    W0[:, 0] = 1.3
    W0[:, D + 1] = 0.7
    out = oracle.run(mesh, Params(solver=meta["solver"], gamma=meta["gamma"]), 1e-3, 3, W0)
    assert out["status"] == 0
    W = out["W"]
    assert np.allclose(W[:, 0], 1.3, rtol=1e-12, atol=0)
    assert np.allclose(W[:, D + 1], 0.7, rtol=1e-12, atol=0)
    assert np.abs(W[:, 1:D + 1]).max() <= 1e-12
