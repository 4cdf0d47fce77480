"""One step of a moving mesh on the GPU (sfx_step_moving, plain FP64):
generator velocities (VorCell::get_velocity with the reflective-box check),
face velocities (VorFace::set_v), fluxes in each face's moving frame and the
drift, against the reference built without -DSTATIC
(tests/golden/moving_*.npz): drifted positions, W and Q bit for bit with
sfx_pow and sfx_cbrt, within 1e-12 per field of the reference with glibc's
pow and cbrt; the case where the reference throws UpdateQException fails
with SFX_ERR_NEG_STATE; the split pass's moving step within 1e-6 of FP64."""
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


@pytest.mark.parametrize("name", MOVING_CASES)
def test_split_moving_step_within_tolerance_of_fp64(cuda_ok, name):
    """the FP32/FP64 split pass with the boost: within 1e-6 relative L1 of the
    plain FP64 moving step per conserved field, the drifted positions within
    1e-9 (the velocities are formed in FP64 from the FP32-rounded state)"""
    mesh, meta, ref = load_case(name)
    ctx, fp = _pass(mesh, meta, precision=1)
    pos = fp.step_moving(meta["dt"], mesh.periodic)
    Q = fp.state()[1]
    Q64 = ref["ref_sfxpow_Q"]
    D = mesh.dim
    den = np.abs(Q64).sum(0)
    den[1:D + 1] = np.sqrt((Q64[:, 1:D + 1] ** 2).sum(1)).sum()
    err = np.abs(Q - Q64).sum(0) / den
    assert np.all(err <= 1e-6), err
    assert np.abs(pos - ref["ref_sfxpow_pos"]).max() <= 1e-9
    assert abs(Q[:, 0].sum() - Q64[:, 0].sum()) <= 1e-13 * Q64[:, 0].sum()
    fp.close()
    ctx.close()


def test_moving_step_is_refused_on_clones(cuda_ok):
    """a clone shares its base's geometry, which a moving step rewrites"""
    from shadowfax_b200 import _lib as L
    mesh, meta, _ = load_case(MOVING_CASES[0])
    ctx, fp = _pass(mesh, meta)
    clone = fp.clone(ctx)
    with pytest.raises(L.SfxError) as ei:
        clone.step_moving(meta["dt"], mesh.periodic)
    assert ei.value.status == L.SFX_ERR_UNSUPPORTED
    clone.close()
    fp.close()
    ctx.close()
