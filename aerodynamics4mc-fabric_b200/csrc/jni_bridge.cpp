// JNI shim: the native methods of the mod's NativeSimulationBridge (brick
// world) and MesoscaleNativeBridge classes, forwarding to this library's C
// ABI. Java declarations: src/main/java/com/aerodynamics4mc/runtime/
// NativeSimulationBridge.java:1239-1656 and MesoscaleNativeBridge.java:129-165;
// the reference's forwarders: native/src/aero_lbm_simulation_bridge.cpp:7026-8985,
// native/src/aero_lbm_mesoscale.cpp:1511-1605, native/src/aero_lbm_jni.cpp:10493-10533.
// Each forwarder checks the Java array lengths as the reference does, pins the
// arrays for the call, releases inputs without copy-back and commits outputs
// only when the call succeeded. The region (server L2), nested-feedback,
// atlas-by-key and codec natives of NativeSimulationBridge are not exported
// (outside the brick path); the JVM reports UnsatisfiedLinkError only if the
// mod calls one of them.
#include <vector>

#include "aero_lbm_b200.h"
#include "jni_abi.h"

using namespace aero_jni;

namespace {

constexpr int kFaceCount = 6;
constexpr int kMesoForcingChannels = 25;
constexpr int kMesoStateChannels = 6;

bool length_is(JNIEnv* env, jarray a, long long n) { return a && n >= 0 && (long long)array_length(env, a) == n; }

jintArray coords_array(JNIEnv* env, int count, bool resident, long long svc, long long world) {
    if (count < 0) return nullptr;
    jintArray out = new_int_array(env, count * 3);
    if (!out || count == 0) return out;
    std::vector<int> coords((size_t)count * 3, 0);
    const int copied = resident ? aero_lbm_simulation_copy_brick_world_resident_bricks(svc, world, coords.data(), count)
                                : aero_lbm_simulation_copy_brick_world_active_bricks(svc, world, coords.data(), count);
    if (copied != count) return nullptr;
    set_int_region(env, out, 0, count * 3, reinterpret_cast<const jint*>(coords.data()));
    return out;
}

void meso_config(AeroLbmMesoscaleConfig& cfg, jint nx, jint ny, jint nz, jfloat dx, jfloat dt, jfloat nu, jfloat pr,
                 jfloat prt) {
    aero_lbm_mesoscale_default_config(&cfg);
    cfg.nx = nx;
    cfg.ny = ny;
    cfg.nz = nz;
    cfg.dx_m = dx;
    cfg.dt_s = dt;
    cfg.molecular_nu_m2_s = nu;
    cfg.prandtl_air = pr;
    cfg.turbulent_prandtl = prt;
}

// static brick upload with or without source fields (both Java signatures)
jboolean upload_static(JNIEnv* env, jlong svc, jlong world, jint n, jint bx, jint by, jint bz, jbyteArray obstacle,
                       jbyteArray surface_kind, jshortArray open_face_mask, jfloatArray emitter, jbyteArray source_fan,
                       jfloatArray source_emitter, jbyteArray sky, jbyteArray direct, bool with_sources, bool queued) {
    const long long cells = (long long)n * n * n;
    if (cells <= 0 || !length_is(env, obstacle, cells) || !length_is(env, surface_kind, cells) ||
        !length_is(env, open_face_mask, cells) || !length_is(env, emitter, cells) || !length_is(env, sky, cells * kFaceCount) ||
        !length_is(env, direct, cells * kFaceCount))
        return JNI_FALSE;
    if (with_sources && (!length_is(env, source_fan, cells) || !length_is(env, source_emitter, cells))) return JNI_FALSE;
    Elements<jbyte> ob(env, obstacle), sk(env, surface_kind), sy(env, sky), di(env, direct);
    Elements<jshort> of(env, open_face_mask);
    Elements<jfloat> em(env, emitter);
    Elements<jbyte> sf(env, with_sources ? source_fan : nullptr);
    Elements<jfloat> se(env, with_sources ? source_emitter : nullptr);
    if (!ob || !sk || !sy || !di || !of || !em || (with_sources && (!sf || !se))) return JNI_FALSE;
    auto u8 = [](const Elements<jbyte>& e) { return reinterpret_cast<const uint8_t*>(e.get()); };
    int ok;
    if (queued) {
        ok = aero_lbm_simulation_queue_brick_world_static_brick_upload(svc, world, n, bx, by, bz, u8(ob), u8(sk),
                                                                       reinterpret_cast<const uint16_t*>(of.get()), em.get(),
                                                                       u8(sy), u8(di));
    } else if (with_sources) {
        ok = aero_lbm_simulation_upload_brick_world_static_brick_with_sources(
            svc, world, n, bx, by, bz, u8(ob), u8(sk), reinterpret_cast<const uint16_t*>(of.get()), em.get(), u8(sf), se.get(),
            u8(sy), u8(di));
    } else {
        ok = aero_lbm_simulation_upload_brick_world_static_brick(svc, world, n, bx, by, bz, u8(ob), u8(sk),
                                                                 reinterpret_cast<const uint16_t*>(of.get()), em.get(), u8(sy),
                                                                 u8(di));
    }
    return ok ? JNI_TRUE : JNI_FALSE;
}

// dynamic / boundary-reference uploads and the dynamic copy-out share their checks
bool dynamic_lengths(JNIEnv* env, jint n, jfloatArray flow, jfloatArray air, jfloatArray surface) {
    const long long cells = (long long)n * n * n;
    return cells > 0 && length_is(env, flow, cells * AERO_LBM_SIMULATION_FLOW_STATE_CHANNELS) && length_is(env, air, cells) &&
           length_is(env, surface, cells);
}

}  // namespace

#define NSB(name) Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_##name
#define MNB(name) Java_com_aerodynamics4mc_runtime_MesoscaleNativeBridge_##name

extern "C" {

// NativeSimulationBridge.java:1239 / simulation_bridge.cpp:7026
AERO_JNIEXPORT jlong AERO_JNICALL NSB(nativeCreateService)(JNIEnv*, jclass) {
    long long key = 0;
    return aero_lbm_simulation_create_service(&key) ? (jlong)key : 0;
}

// NativeSimulationBridge.java:1241 / simulation_bridge.cpp:7031
AERO_JNIEXPORT void AERO_JNICALL NSB(nativeReleaseService)(JNIEnv*, jclass, jlong svc) {
    aero_lbm_simulation_release_service(svc);
}

// NativeSimulationBridge.java:1243 / simulation_bridge.cpp:7039
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeSetFocus)(JNIEnv*, jclass, jlong svc, jint x, jint y, jint z, jint r) {
    return aero_lbm_simulation_set_focus(svc, x, y, z, r) ? JNI_TRUE : JNI_FALSE;
}

// NativeSimulationBridge.java:1245 / simulation_bridge.cpp:7057-7117: 8 ints and
// 4 floats per delta
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeSubmitWorldDeltas)(JNIEnv* env, jclass, jlong svc, jintArray ints,
                                                                  jfloatArray floats) {
    if (!ints || !floats) return JNI_FALSE;
    const jsize ni = array_length(env, ints), nf = array_length(env, floats);
    if (ni % 8 != 0 || nf % 4 != 0 || ni / 8 != nf / 4) return JNI_FALSE;
    const int count = ni / 8;
    Elements<jint> iv(env, ints);
    Elements<jfloat> fv(env, floats);
    if (!iv || !fv) return JNI_FALSE;
    std::vector<AeroLbmWorldDelta> d((size_t)count);
    for (int i = 0; i < count; ++i) {
        const jint* p = iv.get() + 8 * i;
        const jfloat* f = fv.get() + 4 * i;
        d[i] = AeroLbmWorldDelta{p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], f[0], f[1], f[2], f[3]};
    }
    return aero_lbm_simulation_submit_world_deltas(svc, d.data(), count) ? JNI_TRUE : JNI_FALSE;
}

// NativeSimulationBridge.java:1247 / simulation_bridge.cpp:7119
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeEnsureBrickWorldRuntime)(JNIEnv*, jclass, jlong svc, jlong world, jint n,
                                                                        jfloat dx, jfloat dt) {
    return aero_lbm_simulation_ensure_brick_world_runtime(svc, world, n, dx, dt) ? JNI_TRUE : JNI_FALSE;
}

// NativeSimulationBridge.java:1255 / simulation_bridge.cpp:7137
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeSetBrickWorldSolverMode)(JNIEnv*, jclass, jlong svc, jlong world, jint mode) {
    return aero_lbm_simulation_set_brick_world_solver_mode(svc, world, mode) ? JNI_TRUE : JNI_FALSE;
}

static jboolean hints(JNIEnv* env, jlong svc, jlong world, jint n, jintArray coords, jint count, bool exact) {
    if (!coords || count < 0 || (long long)array_length(env, coords) < (long long)count * 3) return JNI_FALSE;
    Elements<jint> c(env, coords);
    if (!c) return JNI_FALSE;
    const int* p = reinterpret_cast<const int*>(c.get());
    const int ok = exact ? aero_lbm_simulation_set_brick_world_exact_active_hints(svc, world, n, p, count)
                         : aero_lbm_simulation_set_brick_world_active_hints(svc, world, n, p, count);
    return ok ? JNI_TRUE : JNI_FALSE;
}

// NativeSimulationBridge.java:1257 / simulation_bridge.cpp:7151
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeSetBrickWorldActiveHints)(JNIEnv* env, jclass, jlong svc, jlong world, jint n,
                                                                         jintArray coords, jint count) {
    return hints(env, svc, world, n, coords, count, false);
}

// NativeSimulationBridge.java:1265 / simulation_bridge.cpp:7182
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeSetBrickWorldExactActiveHints)(JNIEnv* env, jclass, jlong svc, jlong world,
                                                                              jint n, jintArray coords, jint count) {
    return hints(env, svc, world, n, coords, count, true);
}

// NativeSimulationBridge.java:1273 / simulation_bridge.cpp:7213
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeGetBrickWorldRuntimeStatus)(JNIEnv* env, jclass, jlong svc, jlong world,
                                                                           jintArray out) {
    if (!length_is(env, out, AERO_LBM_SIMULATION_BRICK_RUNTIME_STATUS_FIELDS)) return JNI_FALSE;
    Elements<jint> o(env, out);
    if (!o) return JNI_FALSE;
    const int ok = aero_lbm_simulation_get_brick_world_runtime_status(svc, world, reinterpret_cast<int*>(o.get()),
                                                                      AERO_LBM_SIMULATION_BRICK_RUNTIME_STATUS_FIELDS);
    o.commit(ok != 0);
    return ok ? JNI_TRUE : JNI_FALSE;
}

// NativeSimulationBridge.java:1279 / simulation_bridge.cpp:7238
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeStepBrickWorldRuntime)(JNIEnv*, jclass, jlong svc, jlong world, jint steps) {
    return aero_lbm_simulation_step_brick_world_runtime(svc, world, steps) ? JNI_TRUE : JNI_FALSE;
}

// NativeSimulationBridge.java:1285 / simulation_bridge.cpp:7252
AERO_JNIEXPORT jintArray AERO_JNICALL NSB(nativeGetBrickWorldResidentBrickCoords)(JNIEnv* env, jclass, jlong svc, jlong world) {
    return coords_array(env, aero_lbm_simulation_get_brick_world_resident_brick_count(svc, world), true, svc, world);
}

// NativeSimulationBridge.java:1290 / simulation_bridge.cpp:7291
AERO_JNIEXPORT jintArray AERO_JNICALL NSB(nativeGetBrickWorldActiveBrickCoords)(JNIEnv* env, jclass, jlong svc, jlong world) {
    return coords_array(env, aero_lbm_simulation_get_brick_world_active_brick_count(svc, world), false, svc, world);
}

// NativeSimulationBridge.java:1295 / simulation_bridge.cpp:7330
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeUploadBrickWorldStaticBrick)(JNIEnv* env, jclass, jlong svc, jlong world, jint n,
                                                                            jint bx, jint by, jint bz, jbyteArray obstacle,
                                                                            jbyteArray surface_kind, jshortArray open_face_mask,
                                                                            jfloatArray emitter, jbyteArray sky, jbyteArray direct) {
    return upload_static(env, svc, world, n, bx, by, bz, obstacle, surface_kind, open_face_mask, emitter, nullptr, nullptr, sky,
                         direct, false, false);
}

// NativeSimulationBridge.java:1310 / simulation_bridge.cpp:7416
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeUploadBrickWorldStaticBrickWithSources)(
    JNIEnv* env, jclass, jlong svc, jlong world, jint n, jint bx, jint by, jint bz, jbyteArray obstacle, jbyteArray surface_kind,
    jshortArray open_face_mask, jfloatArray emitter, jbyteArray source_fan, jfloatArray source_emitter, jbyteArray sky,
    jbyteArray direct) {
    if (!source_fan || !source_emitter) return JNI_FALSE;
    return upload_static(env, svc, world, n, bx, by, bz, obstacle, surface_kind, open_face_mask, emitter, source_fan,
                         source_emitter, sky, direct, true, false);
}

// NativeSimulationBridge.java:1327 / simulation_bridge.cpp:7506
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeQueueBrickWorldStaticBrickUpload)(JNIEnv* env, jclass, jlong svc, jlong world,
                                                                                 jint n, jint bx, jint by, jint bz,
                                                                                 jbyteArray obstacle, jbyteArray surface_kind,
                                                                                 jshortArray open_face_mask, jfloatArray emitter,
                                                                                 jbyteArray sky, jbyteArray direct) {
    return upload_static(env, svc, world, n, bx, by, bz, obstacle, surface_kind, open_face_mask, emitter, nullptr, nullptr, sky,
                         direct, false, true);
}

// NativeSimulationBridge.java:1360 / simulation_bridge.cpp:7630
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeCopyBrickWorldDynamicBrick)(JNIEnv* env, jclass, jlong svc, jlong world, jint n,
                                                                           jint bx, jint by, jint bz, jfloatArray flow,
                                                                           jfloatArray air, jfloatArray surface) {
    if (!dynamic_lengths(env, n, flow, air, surface)) return JNI_FALSE;
    Elements<jfloat> f(env, flow), a(env, air), s(env, surface);
    if (!f || !a || !s) return JNI_FALSE;
    const int ok = aero_lbm_simulation_copy_brick_world_dynamic_brick(svc, world, n, bx, by, bz, f.get(), a.get(), s.get());
    f.commit(ok != 0);
    a.commit(ok != 0);
    s.commit(ok != 0);
    return ok ? JNI_TRUE : JNI_FALSE;
}

// NativeSimulationBridge.java:1371 / simulation_bridge.cpp:7688-7729
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeCopyBrickWorldPackedFlowAtlas)(JNIEnv* env, jclass, jlong svc, jlong world,
                                                                              jint n, jint bx, jint by, jint bz, jint stride,
                                                                              jshortArray out) {
    if (!out || stride <= 0) return JNI_FALSE;
    const long long res = ((long long)n + stride - 1) / stride;
    const long long values = res * res * res * AERO_LBM_SIMULATION_PACKED_ATLAS_CHANNELS;
    if (res <= 0 || !length_is(env, out, values)) return JNI_FALSE;
    Elements<jshort> o(env, out);
    if (!o) return JNI_FALSE;
    const int ok = aero_lbm_simulation_copy_brick_world_packed_flow_atlas(svc, world, n, bx, by, bz, stride,
                                                                          reinterpret_cast<int16_t*>(o.get()), (int)values);
    o.commit(ok != 0);
    return ok ? JNI_TRUE : JNI_FALSE;
}

// NativeSimulationBridge.java:1381 / simulation_bridge.cpp:7731
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeUploadBrickWorldDynamicBrick)(JNIEnv* env, jclass, jlong svc, jlong world,
                                                                             jint n, jint bx, jint by, jint bz, jfloatArray flow,
                                                                             jfloatArray air, jfloatArray surface) {
    if (!dynamic_lengths(env, n, flow, air, surface)) return JNI_FALSE;
    Elements<jfloat> f(env, flow), a(env, air), s(env, surface);
    if (!f || !a || !s) return JNI_FALSE;
    return aero_lbm_simulation_upload_brick_world_dynamic_brick(svc, world, n, bx, by, bz, f.get(), a.get(), s.get())
               ? JNI_TRUE
               : JNI_FALSE;
}

// NativeSimulationBridge.java:1392 / simulation_bridge.cpp:7789
AERO_JNIEXPORT jboolean AERO_JNICALL NSB(nativeUploadBrickWorldBoundaryReferenceBrick)(JNIEnv* env, jclass, jlong svc,
                                                                                       jlong world, jint n, jint bx, jint by,
                                                                                       jint bz, jfloatArray flow,
                                                                                       jfloatArray air, jfloatArray surface) {
    if (!dynamic_lengths(env, n, flow, air, surface)) return JNI_FALSE;
    Elements<jfloat> f(env, flow), a(env, air), s(env, surface);
    if (!f || !a || !s) return JNI_FALSE;
    return aero_lbm_simulation_upload_brick_world_boundary_reference_brick(svc, world, n, bx, by, bz, f.get(), a.get(), s.get())
               ? JNI_TRUE
               : JNI_FALSE;
}

// NativeSimulationBridge.java:1654-1656 / simulation_bridge.cpp:8977-8983
AERO_JNIEXPORT jstring AERO_JNICALL NSB(nativeRuntimeInfo)(JNIEnv* env, jclass) {
    return new_string_utf(env, aero_lbm_simulation_runtime_info());
}
AERO_JNIEXPORT jstring AERO_JNICALL NSB(nativeLastError)(JNIEnv* env, jclass) {
    return new_string_utf(env, aero_lbm_simulation_last_error());
}

// MesoscaleNativeBridge.java:129 / aero_lbm_jni.cpp:10493-10533: transport as
// float[5] (velocity scale, nu, alpha, tau shear, tau thermal)
AERO_JNIEXPORT jfloatArray AERO_JNICALL MNB(nativeDeriveTransport)(JNIEnv* env, jclass, jint nx, jint ny, jint nz, jfloat dx,
                                                                   jfloat dt, jfloat nu, jfloat pr, jfloat prt) {
    AeroLbmMesoscaleConfig cfg{};
    meso_config(cfg, nx, ny, nz, dx, dt, nu, pr, prt);
    AeroLbmMesoscaleTransport t{};
    if (!aero_lbm_mesoscale_derive_transport(&cfg, &t)) return nullptr;
    jfloatArray out = new_float_array(env, 5);
    if (!out) return nullptr;
    const jfloat v[5] = {t.velocity_scale_m_s_per_lattice, t.nu_molecular_lattice, t.alpha_molecular_lattice,
                         t.tau_shear_molecular, t.tau_thermal_molecular};
    set_float_region(env, out, 0, 5, v);
    return out;
}

// MesoscaleNativeBridge.java:140 / aero_lbm_mesoscale.cpp:1511-1535
AERO_JNIEXPORT jlong AERO_JNICALL MNB(nativeCreateContext)(JNIEnv*, jclass, jint nx, jint ny, jint nz, jfloat dx, jfloat dt,
                                                           jfloat nu, jfloat pr, jfloat prt) {
    AeroLbmMesoscaleConfig cfg{};
    meso_config(cfg, nx, ny, nz, dx, dt, nu, pr, prt);
    long long key = 0;
    return aero_lbm_mesoscale_create_context(&cfg, &key) ? (jlong)key : 0;
}

// MesoscaleNativeBridge.java:151 / aero_lbm_mesoscale.cpp:1537-1595: the
// state array is written back whether or not the step succeeded
AERO_JNIEXPORT jboolean AERO_JNICALL MNB(nativeStepContext)(JNIEnv* env, jclass, jlong key, jint nx, jint ny, jint nz,
                                                            jfloat dx, jfloat dt, jfloat nu, jfloat pr, jfloat prt,
                                                            jfloatArray forcing, jfloatArray out_state) {
    if (!forcing || !out_state) return JNI_FALSE;
    AeroLbmMesoscaleConfig cfg{};
    meso_config(cfg, nx, ny, nz, dx, dt, nu, pr, prt);
    const long long cells = (long long)cfg.nx * cfg.ny * cfg.nz;
    if (!length_is(env, forcing, cells * kMesoForcingChannels) || !length_is(env, out_state, cells * kMesoStateChannels))
        return JNI_FALSE;
    Elements<jfloat> f(env, forcing), o(env, out_state);
    o.commit(true);
    if (!f || !o) return JNI_FALSE;
    return aero_lbm_mesoscale_step_context(key, &cfg, f.get(), o.get()) ? JNI_TRUE : JNI_FALSE;
}

// MesoscaleNativeBridge.java:165 / aero_lbm_mesoscale.cpp:1597-1603
AERO_JNIEXPORT void AERO_JNICALL MNB(nativeReleaseContext)(JNIEnv*, jclass, jlong key) {
    aero_lbm_mesoscale_release_context(key);
}

}  // extern "C"
