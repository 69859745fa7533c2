"""The brick-world service (aero_lbm_simulation_*) and its JNI shim, on the
CPU: everything the service does before a brick steps (worlds, hints,
static uploads with their source fields, dynamic uploads with the static
constraints, boundary references, the packed atlas of a brick that has not
stepped, status, coordinate lists, world deltas queued for the next step,
argument errors) against the reference's own service
(oracle/_ref/libaero_sim_ref.so, built from its sources), bit for bit; and
the JNI forwarders called through a fake JNIEnv whose function table sits at
the JNI specification's indices."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import aero_b200
import oracle as O

ROOT = Path(__file__).resolve().parents[1]


def _host_only(script):
    """The operations of a script up to its first step (no device needed)."""
    out = []
    for op in script:
        if op[0] == "step":
            break
        out.append(op)
    return out


def _host_script(n=12):
    s = _host_only(O.brick_world_rich_script(n=n))
    W = 1
    bricks = [(0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 0, 1), (1, 0, 1)]
    s += [("status", W), ("coords", W, True), ("coords", W, False)]
    s += [("copy", W, n, b) for b in bricks] + [("atlas", W, n, b, st) for b in bricks for st in (1, 3, 4, 5)]
    # errors: wrong brick size, unknown world, wrong atlas size are rejected alike
    s += [("atlas", W, n + 1, (0, 0, 0), 4), ("copy", 7, n, (0, 0, 0)), ("status", 7), ("mode", 7, 1)]
    s += [("deltas", [(8, 6, 5, 6, W, 0x1, 0, 0, 0.0, 0.0, 0.0, 0.0), (4, 0, 0, 0, W, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)]),
          ("status", W)]
    # a world reset by a new brick size drops its bricks
    s += [("ensure", W, n // 2, 1.0, 0.05), ("status", W), ("coords", W, True)]
    return s


def _compare(a, b):
    assert len(a) == len(b)
    for i, (x, y) in enumerate(zip(a, b)):
        assert x[0] == y[0], (i, x[0], y[0])
        for u, v in zip(x[1:], y[1:]):
            if isinstance(u, np.ndarray):
                assert u.dtype == v.dtype and np.array_equal(u.view(np.uint8), v.view(np.uint8)), (i, x[0])
            else:
                assert u == v, (i, x, y)


@pytest.mark.skipif(not O.SIM_REF_LIB.exists(), reason="reference service not built (make -C oracle sim)")
def test_host_bookkeeping_matches_reference_service(lib):
    script = _host_script()
    ref = O.run_brick_script(O.SIM_REF_LIB, script)
    ours = O.run_brick_script(aero_b200.LIB_PATH, script)
    _compare(ref, ours)
    # the uploads were constrained: obstacle cells read back as zeros
    copies = [r for r in ours if r[0] == "copy" and r[1] == 1]
    assert copies and all(np.isfinite(c[2]).all() for c in copies)


def test_service_argument_errors(lib):
    svc = aero_b200.BrickWorldService(lib)
    try:
        with pytest.raises(RuntimeError, match="invalid runtime config"):
            svc.ensure_world(3, 8, dx=0.0)
        svc.ensure_world(3, 8)
        assert lib.aero_lbm_simulation_step_brick_world_runtime(svc.key, 3, 0) == 0
        assert "invalid step count" in svc.error()
        assert lib.aero_lbm_simulation_step_brick_world_runtime(svc.key, 99, 1) == 0
        assert "missing brick runtime" in svc.error()
        st = np.zeros(4, np.int32)
        assert lib.aero_lbm_simulation_get_brick_world_runtime_status(
            svc.key, 3, st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 4) == 0
        assert "invalid output buffer" in svc.error()
        assert lib.aero_lbm_simulation_set_brick_world_solver_mode(svc.key + 5, 3, 1) == 0
        assert "missing service" in svc.error()
    finally:
        svc.release()


# ---------------------------------------------------------------- JNI shim
JNI_SLOTS = {"NewStringUTF": 167, "GetArrayLength": 171, "NewIntArray": 179, "NewFloatArray": 181,
             "GetByteArrayElements": 184, "GetShortArrayElements": 186, "GetIntArrayElements": 187,
             "GetFloatArrayElements": 189, "ReleaseByteArrayElements": 192, "ReleaseShortArrayElements": 194,
             "ReleaseIntArrayElements": 195, "ReleaseFloatArrayElements": 197, "SetIntArrayRegion": 211,
             "SetFloatArrayRegion": 213}
JNI_ABORT = 2


class FakeJVM:
    """A JNIEnv whose array elements are copies (as a JVM may hand out):
    Release with mode 0 copies back, JNI_ABORT discards."""

    def __init__(self):
        self.objects: dict[int, object] = {}
        self.pinned: dict[int, tuple[int, np.ndarray]] = {}
        self.released_modes: list[int] = []
        self.next = 1
        vp, i32 = ctypes.c_void_p, ctypes.c_int32
        self._cbs = []
        table = (ctypes.c_void_p * 235)()

        def put(name, restype, argtypes, fn):
            cb = ctypes.CFUNCTYPE(restype, *argtypes)(fn)
            self._cbs.append(cb)
            table[JNI_SLOTS[name]] = ctypes.cast(cb, ctypes.c_void_p)

        put("GetArrayLength", i32, [vp, vp], lambda env, a: int(self.objects[a].size))
        for name in ("Byte", "Short", "Int", "Float"):
            put(f"Get{name}ArrayElements", vp, [vp, vp, vp], self._get)
            put(f"Release{name}ArrayElements", None, [vp, vp, vp, i32], self._release)
        put("NewIntArray", vp, [vp, i32], lambda env, n: self.new(np.zeros(n, np.int32)))
        put("NewFloatArray", vp, [vp, i32], lambda env, n: self.new(np.zeros(n, np.float32)))
        put("SetIntArrayRegion", None, [vp, vp, i32, i32, vp], self._set_region)
        put("SetFloatArrayRegion", None, [vp, vp, i32, i32, vp], self._set_region)
        put("NewStringUTF", vp, [vp, ctypes.c_char_p], lambda env, s: self.new(s.decode()))
        self.table = table
        self.env_ptr = ctypes.c_void_p(ctypes.addressof(table))
        self.env = ctypes.byref(self.env_ptr)

    def new(self, obj) -> int:
        h = self.next
        self.next += 1
        self.objects[h] = obj
        return h

    def _get(self, env, a, is_copy):
        copy = np.array(self.objects[a], copy=True)
        addr = copy.ctypes.data
        self.pinned[addr] = (a, copy)
        return addr

    def _release(self, env, a, ptr, mode):
        handle, copy = self.pinned.pop(ptr)
        assert handle == a
        self.released_modes.append(mode)
        if mode != JNI_ABORT:
            self.objects[a][...] = copy

    def _set_region(self, env, a, start, n, buf):
        dst = self.objects[a]
        src = np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(np.ctypeslib.as_ctypes_type(dst.dtype))), (n,))
        dst[start:start + n] = src


def _jni(lib, name, restype, *argtypes):
    fn = getattr(lib, name)
    fn.restype = restype
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, *argtypes]
    return fn


def test_jni_symbols_declared_and_exported():
    header = (ROOT / "include" / "aero_lbm_b200_jni.h").read_text()
    declared = set(re.findall(r"\b(Java_com_aerodynamics4mc_runtime_\w+)\s*\(", header))
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", str(aero_b200.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T Java_" in line}
    assert len(declared) >= 25 and declared == exported


def test_jni_forwarders_through_fake_env(lib):
    jvm = FakeJVM()
    env = jvm.env
    vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    P = "Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_"
    create = _jni(lib, P + "nativeCreateService", i64)
    ensure = _jni(lib, P + "nativeEnsureBrickWorldRuntime", ctypes.c_uint8, i64, i64, i32, f32, f32)
    hints = _jni(lib, P + "nativeSetBrickWorldExactActiveHints", ctypes.c_uint8, i64, i64, i32, vp, i32)
    upload = _jni(lib, P + "nativeUploadBrickWorldStaticBrickWithSources", ctypes.c_uint8, i64, i64, i32, i32, i32, i32,
                  *([vp] * 8))
    dyn = _jni(lib, P + "nativeUploadBrickWorldDynamicBrick", ctypes.c_uint8, i64, i64, i32, i32, i32, i32, vp, vp, vp)
    status = _jni(lib, P + "nativeGetBrickWorldRuntimeStatus", ctypes.c_uint8, i64, i64, vp)
    copy = _jni(lib, P + "nativeCopyBrickWorldDynamicBrick", ctypes.c_uint8, i64, i64, i32, i32, i32, i32, vp, vp, vp)
    atlas = _jni(lib, P + "nativeCopyBrickWorldPackedFlowAtlas", ctypes.c_uint8, i64, i64, i32, i32, i32, i32, i32, vp)
    coords = _jni(lib, P + "nativeGetBrickWorldActiveBrickCoords", vp, i64, i64)
    last_error = _jni(lib, P + "nativeLastError", vp)
    deltas = _jni(lib, P + "nativeSubmitWorldDeltas", ctypes.c_uint8, i64, vp, vp)
    release = _jni(lib, P + "nativeReleaseService", None, i64)

    n, W = 8, 4
    cells = n ** 3
    svc = create(env, None)
    assert svc == 1
    assert ensure(env, None, svc, W, n, 1.0, 0.05) == 1
    assert hints(env, None, svc, W, n, jvm.new(np.array([0, 0, 0, 1, 0, 0], np.int32)), 2) == 1
    rng = np.random.default_rng(3)
    ob = (rng.random(cells) < 0.2).astype(np.int8)
    arrays = [jvm.new(ob), jvm.new(np.zeros(cells, np.int8)), jvm.new(np.zeros(cells, np.int16)),
              jvm.new(np.zeros(cells, np.float32)), jvm.new(np.zeros(cells, np.int8)), jvm.new(np.zeros(cells, np.float32)),
              jvm.new(np.zeros(cells * 6, np.int8)), jvm.new(np.zeros(cells * 6, np.int8))]
    assert upload(env, None, svc, W, n, 0, 0, 0, *arrays) == 1
    flow = rng.uniform(-0.05, 0.05, cells * 4).astype(np.float32)
    air = rng.uniform(-0.1, 0.1, cells).astype(np.float32)
    assert dyn(env, None, svc, W, n, 0, 0, 0, jvm.new(flow), jvm.new(air), jvm.new(np.zeros(cells, np.float32))) == 1

    st = jvm.new(np.full(8, -1, np.int32))
    assert status(env, None, svc, W, st) == 1
    assert jvm.objects[st].tolist() == [n, 2, 2, 1, 1, 0, 0, 1]  # committed back (mode 0)
    # the copy-out is the upload with obstacle cells zeroed
    out_f, out_a, out_s = (jvm.new(np.zeros(cells * 4, np.float32)), jvm.new(np.zeros(cells, np.float32)),
                           jvm.new(np.zeros(cells, np.float32)))
    assert copy(env, None, svc, W, n, 0, 0, 0, out_f, out_a, out_s) == 1
    expect = flow.reshape(-1, 4).copy()
    expect[ob != 0] = 0
    assert np.array_equal(jvm.objects[out_f].reshape(-1, 4), expect)
    a_out = jvm.new(np.zeros(2 ** 3 * 4, np.int16))
    assert atlas(env, None, svc, W, n, 0, 0, 0, 4, a_out) == 1
    assert np.any(jvm.objects[a_out] != 0)
    # a wrong-length output is rejected before the call, a failed call
    # releases its output without copy-back
    assert atlas(env, None, svc, W, n, 0, 0, 0, 4, jvm.new(np.zeros(7, np.int16))) == 0
    st_bad = jvm.new(np.full(8, -1, np.int32))
    assert status(env, None, svc, 99, st_bad) == 0
    assert jvm.objects[st_bad].tolist() == [-1] * 8
    msg = last_error(env, None)
    assert "missing brick runtime" in jvm.objects[msg]
    c = coords(env, None, svc, W)
    assert jvm.objects[c].tolist() == [0, 0, 0]
    assert deltas(env, None, svc, jvm.new(np.zeros(8, np.int32)), jvm.new(np.zeros(3, np.float32))) == 0
    assert deltas(env, None, svc, jvm.new(np.array([4, 0, 0, 0, W, 0, 0, 0], np.int32)),
                  jvm.new(np.zeros(4, np.float32))) == 1
    release(env, None, svc)
    assert not jvm.pinned, "every pinned array was released"
    assert JNI_ABORT in jvm.released_modes and 0 in jvm.released_modes


def test_jni_mesoscale_transport(lib):
    jvm = FakeJVM()
    vp, i32, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_float
    derive = _jni(lib, "Java_com_aerodynamics4mc_runtime_MesoscaleNativeBridge_nativeDeriveTransport", vp,
                  i32, i32, i32, f32, f32, f32, f32, f32)
    h = derive(jvm.env, None, 16, 8, 16, 64.0, 5.0, 1.5e-5, 0.71, 0.85)
    got = jvm.objects[h]
    cfg = aero_b200.AeroLbmMesoscaleConfig()
    lib.aero_lbm_mesoscale_default_config(ctypes.byref(cfg))
    cfg.nx, cfg.ny, cfg.nz, cfg.dx_m, cfg.dt_s = 16, 8, 16, 64.0, 5.0
    cfg.molecular_nu_m2_s, cfg.prandtl_air, cfg.turbulent_prandtl = 1.5e-5, 0.71, 0.85
    t = aero_b200.AeroLbmMesoscaleTransport()
    assert lib.aero_lbm_mesoscale_derive_transport(ctypes.byref(cfg), ctypes.byref(t)) == 1
    assert got.tolist() == np.array([t.velocity_scale_m_s_per_lattice, t.nu_molecular_lattice, t.alpha_molecular_lattice,
                                     t.tau_shear_molecular, t.tau_thermal_molecular], np.float32).tolist()
