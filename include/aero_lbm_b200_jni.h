/*
 * aero_lbm_b200_jni — the JNI native methods libaero_lbm_b200.so exports for
 * the mod's Java bridges, so that the mod's NativeLibraryLoader can load this
 * library in place of the reference's (the JVM binds a `native` method to the
 * exported symbol named Java_<class>_<method>).
 *
 * Java side: com.aerodynamics4mc.runtime.NativeSimulationBridge
 * (src/main/java/com/aerodynamics4mc/runtime/NativeSimulationBridge.java:1239-1656)
 * and com.aerodynamics4mc.runtime.MesoscaleNativeBridge
 * (src/main/java/com/aerodynamics4mc/runtime/MesoscaleNativeBridge.java:129-165).
 * Each symbol replaces the reference forwarder cited beside it and forwards
 * to the C ABI of aero_lbm_b200.h. JNI types are spelled with their
 * fixed-width C equivalents: JNIEnv* and jclass/jarray/jstring handles as
 * void*, jboolean uint8_t, jint int32_t, jlong int64_t, jfloat float.
 */
#ifndef AERO_LBM_B200_JNI_H
#define AERO_LBM_B200_JNI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* native/src/aero_lbm_simulation_bridge.cpp:7026 */
int64_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeCreateService(void* env, void* cls);
/* :7031 */
void Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeReleaseService(void* env, void* cls, int64_t service);
/* :7039 */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeSetFocus(void* env, void* cls, int64_t service,
                                                                              int32_t x, int32_t y, int32_t z, int32_t radius);
/* :7057 (int[8 * n] deltas, float[4 * n] values) */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeSubmitWorldDeltas(void* env, void* cls, int64_t service,
                                                                                       void* ints, void* floats);
/* :7119 */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeEnsureBrickWorldRuntime(
    void* env, void* cls, int64_t service, int64_t world, int32_t brick_size, float dx, float dt);
/* :7137 */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeSetBrickWorldSolverMode(void* env, void* cls,
                                                                                             int64_t service, int64_t world,
                                                                                             int32_t mode);
/* :7151, :7182 (int[3 * count] brick coordinates) */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeSetBrickWorldActiveHints(
    void* env, void* cls, int64_t service, int64_t world, int32_t brick_size, void* coords, int32_t count);
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeSetBrickWorldExactActiveHints(
    void* env, void* cls, int64_t service, int64_t world, int32_t brick_size, void* coords, int32_t count);
/* :7213 (int[8]) */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeGetBrickWorldRuntimeStatus(
    void* env, void* cls, int64_t service, int64_t world, void* out_status);
/* :7238 */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeStepBrickWorldRuntime(void* env, void* cls,
                                                                                           int64_t service, int64_t world,
                                                                                           int32_t steps);
/* :7252, :7291 (returns int[3 * n]) */
void* Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeGetBrickWorldResidentBrickCoords(void* env, void* cls,
                                                                                                    int64_t service,
                                                                                                    int64_t world);
void* Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeGetBrickWorldActiveBrickCoords(void* env, void* cls,
                                                                                                  int64_t service,
                                                                                                  int64_t world);
/* :7330, :7416, :7506 (byte[n^3] obstacle, byte[n^3] surface kind, short[n^3]
 * open faces, float[n^3] emitter power, [byte[n^3] source fan dir, float[n^3]
 * source emitter power,] byte[6 n^3] sky and direct exposure) */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeUploadBrickWorldStaticBrick(
    void* env, void* cls, int64_t service, int64_t world, int32_t brick_size, int32_t bx, int32_t by, int32_t bz,
    void* obstacle, void* surface_kind, void* open_face_mask, void* emitter, void* sky, void* direct);
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeUploadBrickWorldStaticBrickWithSources(
    void* env, void* cls, int64_t service, int64_t world, int32_t brick_size, int32_t bx, int32_t by, int32_t bz,
    void* obstacle, void* surface_kind, void* open_face_mask, void* emitter, void* source_fan, void* source_emitter,
    void* sky, void* direct);
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeQueueBrickWorldStaticBrickUpload(
    void* env, void* cls, int64_t service, int64_t world, int32_t brick_size, int32_t bx, int32_t by, int32_t bz,
    void* obstacle, void* surface_kind, void* open_face_mask, void* emitter, void* sky, void* direct);
/* :7630 (float[4 n^3] flow, float[n^3] air and surface temperature) */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeCopyBrickWorldDynamicBrick(
    void* env, void* cls, int64_t service, int64_t world, int32_t brick_size, int32_t bx, int32_t by, int32_t bz,
    void* flow, void* air, void* surface);
/* :7688 (short[4 ceil(n / stride)^3]) */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeCopyBrickWorldPackedFlowAtlas(
    void* env, void* cls, int64_t service, int64_t world, int32_t brick_size, int32_t bx, int32_t by, int32_t bz,
    int32_t stride, void* out);
/* :7731, :7789 */
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeUploadBrickWorldDynamicBrick(
    void* env, void* cls, int64_t service, int64_t world, int32_t brick_size, int32_t bx, int32_t by, int32_t bz,
    void* flow, void* air, void* surface);
uint8_t Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeUploadBrickWorldBoundaryReferenceBrick(
    void* env, void* cls, int64_t service, int64_t world, int32_t brick_size, int32_t bx, int32_t by, int32_t bz,
    void* flow, void* air, void* surface);
/* :8977, :8981 (return java.lang.String) */
void* Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeRuntimeInfo(void* env, void* cls);
void* Java_com_aerodynamics4mc_runtime_NativeSimulationBridge_nativeLastError(void* env, void* cls);

/* native/src/aero_lbm_jni.cpp:10493 (returns float[5]) */
void* Java_com_aerodynamics4mc_runtime_MesoscaleNativeBridge_nativeDeriveTransport(void* env, void* cls, int32_t nx,
                                                                                   int32_t ny, int32_t nz, float dx, float dt,
                                                                                   float nu, float prandtl,
                                                                                   float turbulent_prandtl);
/* native/src/aero_lbm_mesoscale.cpp:1511 */
int64_t Java_com_aerodynamics4mc_runtime_MesoscaleNativeBridge_nativeCreateContext(void* env, void* cls, int32_t nx,
                                                                                  int32_t ny, int32_t nz, float dx, float dt,
                                                                                  float nu, float prandtl,
                                                                                  float turbulent_prandtl);
/* :1537 (float[25 cells] forcing, float[6 cells] state) */
uint8_t Java_com_aerodynamics4mc_runtime_MesoscaleNativeBridge_nativeStepContext(void* env, void* cls, int64_t key,
                                                                                int32_t nx, int32_t ny, int32_t nz, float dx,
                                                                                float dt, float nu, float prandtl,
                                                                                float turbulent_prandtl, void* forcing,
                                                                                void* out_state);
/* :1597 */
void Java_com_aerodynamics4mc_runtime_MesoscaleNativeBridge_nativeReleaseContext(void* env, void* cls, int64_t key);

#ifdef __cplusplus
}
#endif

#endif
