"""mfdm_step_noalloc, the entry point for callers that cannot allocate device
memory, against the handle-based entry point (mfdm_open_desc + mfdm_step) and
the CPU oracle.

The test owns every device buffer (torch allocates them); the entry point only
uses its static array. Two calls in a row: the second continues the first
(time index and ADE memory), as a caller's time loop would. Both entry points
build their Ricker and PML tables with the same host functions, so their
wavefields are bit-identical. Collected last, so a run that stops at the first
failure has run everything else before it."""
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
        assert np.array_equal(got, ref1[field]), (name, "first call, bitwise")
    mfdm.step_noalloc(dm, n1, n2)
    for name, field in STATE_TO_FIELD.items():
        got = state[name].cpu().numpy()
        assert rel_l2(got, ref2[field]) <= TOL, (name, "second call")
        assert np.array_equal(got, ref2[field]), (name, "second call, bitwise")
    assert np.abs(state["p_f"].cpu().numpy()).max() > 0


def test_noalloc_matches_oracle(mfdm, oracle, cases):
    """Two calls against the FP32 CPU oracle's wavefield after the same steps."""
    import torch
    mfdm.build()
    model = cases.curv_small()
    n1, n2 = 37, 45
    dm, state, keep = _device_model(mfdm, model, torch)
    mfdm.step_noalloc(dm, 0, n1)
    mfdm.step_noalloc(dm, n1, n2)
    ref = oracle.forward(model, n1 + n2, oracle.record_gap(model.dt), 32, final_fields=True)
    for q, name in enumerate(("vx_f", "vz_f", "p_f")):
        assert rel_l2(state[name].cpu().numpy(), ref["fluid"][q]) <= TOL, name
    for q, name in enumerate(("vx_s", "vz_s", "sx_s", "sz_s", "sxz_s")):
        assert rel_l2(state[name].cpu().numpy(), ref["solid"][q]) <= TOL, name


def test_noalloc_long_call_crosses_ricker_table_chunks(mfdm, cases):
    """A call of more steps than the fixed Ricker table holds (1024) refills the
    table between chunks; a 5 Hz wavelet is still non-zero across the refill."""
    import torch
    mfdm.build()
    model = cases.curv_small()
    model.fpeak = 5.0  # Ricker non-zero until 2.4 / 5 Hz = 0.48 s = step 1200
    n = 1100
    with mfdm.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        s.step(n)
        ref = {f: s.field(f) for f in STATE_TO_FIELD.values()}
    dm, state, keep = _device_model(mfdm, model, torch)
    mfdm.step_noalloc(dm, 0, n)
    for name, field in STATE_TO_FIELD.items():
        assert np.array_equal(state[name].cpu().numpy(), ref[field]), name


def test_noalloc_rejects_a_source_outside_the_grid(mfdm, cases):
    import torch
    mfdm.build()
    model = cases.curv_small()
    dm, state, keep = _device_model(mfdm, model, torch)
    dm.src_z = model.nz_f  # one row below the fluid
    with pytest.raises(mfdm.MfdmError) as ei:
        mfdm.step_noalloc(dm, 0, 1)
    assert ei.value.code == -1 and "source outside" in str(ei.value)


def test_noalloc_rejects_models_over_the_static_limit(mfdm, modelgen):
    import torch
    mfdm.build()
    model = modelgen.curvilinear_1200x800(nt=10)
    dm, state, keep = _device_model(mfdm, model, torch)
    with pytest.raises(mfdm.MfdmError) as ei:
        mfdm.step_noalloc(dm, 0, 1)
    assert ei.value.code == -1 and "static limit" in str(ei.value)
