"""One step of a moving mesh on the GPU (sfx_step_moving, plain FP64):
generator velocities (VorCell::get_velocity with the reflective-box check),
face velocities (VorFace::set_v), fluxes in each face's moving frame and the
drift, against the reference built without -DSTATIC
(tests/golden/moving_*.npz): drifted positions, W and Q bit for bit with
sfx_pow and sfx_cbrt, within 1e-12 per field of the reference with glibc's
pow and cbrt; the case where the reference throws UpdateQException fails
with SFX_ERR_NEG_STATE."""
import numpy as np
import pytest

from golden_util import MOVING_CASES, MOVING_FAILS, load_case

pytestmark = pytest.mark.gpu


def _pass(mesh, meta, precision=0):
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    ctx = Context(mesh.dim, RiemannSolverFactory.generate(meta["solver"], meta["gamma"]),
                  precision)
    fp = FluxPass(ctx, mesh)
    fp.set_primitive(meta["W0"])
    return ctx, fp


@pytest.mark.parametrize("name", MOVING_CASES)
def test_moving_step_bitwise_vs_reference(cuda_ok, name):
    mesh, meta, ref = load_case(name)
    ctx, fp = _pass(mesh, meta)
    pos = fp.step_moving(meta["dt"], mesh.periodic)
    W, Q = fp.state()
    np.testing.assert_array_equal(pos, ref["ref_sfxpow_pos"])
    np.testing.assert_array_equal(Q, ref["ref_sfxpow_Q"])
    np.testing.assert_array_equal(W, ref["ref_sfxpow_W"])
    b = ref["ref_libm_Q"]
    for k in range(b.shape[1]):
        lim = 1e-12 * np.abs(b[:, k]) + 1e-15 * np.abs(b[:, k]).max()
        assert np.all(np.abs(Q[:, k] - b[:, k]) <= lim), k
    fp.close()
    ctx.close()


def test_moving_step_fails_where_the_reference_fails(cuda_ok):
    from shadowfax_b200 import _lib as L
    mesh, meta, ref = load_case(MOVING_FAILS)
    ctx, fp = _pass(mesh, meta)
    with pytest.raises(L.SfxError) as ei:
        fp.step_moving(meta["dt"], mesh.periodic)
    assert ei.value.status == L.SFX_ERR_NEG_STATE
    fp.close()
    ctx.close()


def test_moving_step_is_refused_where_unsupported(cuda_ok):
    """split precision and clones share or lack what a moving step rewrites"""
    from shadowfax_b200 import _lib as L
    mesh, meta, _ = load_case(MOVING_CASES[0])
    ctx, fp = _pass(mesh, meta, precision=1)
    with pytest.raises(L.SfxError) as ei:
        fp.step_moving(meta["dt"], mesh.periodic)
    assert ei.value.status == L.SFX_ERR_UNSUPPORTED
    fp.close()
    ctx.close()
    ctx, fp = _pass(mesh, meta)
    clone = fp.clone(ctx)
    with pytest.raises(L.SfxError) as ei:
        clone.step_moving(meta["dt"], mesh.periodic)
    assert ei.value.status == L.SFX_ERR_UNSUPPORTED
    clone.close()
    fp.close()
    ctx.close()
