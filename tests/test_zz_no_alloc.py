"""mfdm_step_noalloc, the entry point for callers that cannot allocate device
memory, against the handle-based entry point (mfdm_open_desc + mfdm_step).

The test owns every device buffer (torch allocates them); the entry point only
uses its static array. Two calls in a row: the second continues the first
(time index and ADE memory), as a caller's time loop would. Collected last, so
a run that stops at the first failure has run everything else before it."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _device_model(mfdm, model, torch):
    keep = {}

    def dev(a):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()
        keep[id(t)] = t
        return t

    dm = mfdm.DeviceModel()
    dm.nx, dm.nz_f, dm.nz_s = model.nx, model.nz_f, model.nz_s
    dm.fpeak, dm.dt, dm.npd, dm.npow = model.fpeak, model.dt, model.npd, model.npow
    dm.thickness, dm.vp_max, dm.rc, dm.beta0 = model.thickness, model.vp_max, model.rc, model.beta0
    dm.src_x, dm.src_z = model.src_x[0], model.src_z[0]
    for name, arr in (("K", model.fluid["K"]), ("rho_f", model.fluid["rho"]),
                      ("C11", model.solid["C11"]), ("C13", model.solid["C13"]),
                      ("C33", model.solid["C33"]), ("C55", model.solid["C55"]),
                      ("rho_s", model.solid["rho"]), ("J", model.metric["J"]),
                      ("xi_x", model.metric["xi_x"]), ("xi_z", model.metric["xi_z"]),
                      ("ze_x", model.metric["ze_x"]), ("ze_z", model.metric["ze_z"])):
        setattr(dm, name, dev(arr).data_ptr())
    state = {}
    for name, rows in (("vx_f", model.nz_f), ("vz_f", model.nz_f), ("p_f", model.nz_f),
                       ("vx_s", model.nz_s), ("vz_s", model.nz_s), ("sx_s", model.nz_s),
                       ("sz_s", model.nz_s), ("sxz_s", model.nz_s)):
        t = torch.zeros((rows, model.nx), dtype=torch.float32, device="cuda")
        state[name] = t
        setattr(dm, name, t.data_ptr())
    return dm, state, keep


STATE_TO_FIELD = {"vx_f": "fluid_vx", "vz_f": "fluid_vz", "p_f": "fluid_p", "vx_s": "solid_vx",
                  "vz_s": "solid_vz", "sx_s": "solid_sx", "sz_s": "solid_sz", "sxz_s": "solid_sxz"}


def test_noalloc_matches_handle_path_over_two_calls(mfdm, cases):
    import torch
    mfdm.build()
    model = cases.curv_small()
    n1, n2 = 37, 45  # odd first chunk: the second call starts on a B-first step
    with mfdm.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        s.step(n1)
        ref1 = {f: s.field(f) for f in STATE_TO_FIELD.values()}
        s.step(n2)
        ref2 = {f: s.field(f) for f in STATE_TO_FIELD.values()}
    dm, state, keep = _device_model(mfdm, model, torch)
    mfdm.step_noalloc(dm, 0, n1)
    for name, field in STATE_TO_FIELD.items():
        got = state[name].cpu().numpy()
        assert rel_l2(got, ref1[field]) <= TOL, (name, "first call")
    mfdm.step_noalloc(dm, n1, n2)
    for name, field in STATE_TO_FIELD.items():
        got = state[name].cpu().numpy()
        assert rel_l2(got, ref2[field]) <= TOL, (name, "second call")
    assert np.abs(state["p_f"].cpu().numpy()).max() > 0


def test_noalloc_rejects_models_over_the_static_limit(mfdm, modelgen):
    import torch
    mfdm.build()
    model = modelgen.curvilinear_1200x800(nt=10)
    dm, state, keep = _device_model(mfdm, model, torch)
    with pytest.raises(mfdm.MfdmError) as ei:
        mfdm.step_noalloc(dm, 0, 1)
    assert ei.value.code == -1 and "static limit" in str(ei.value)
