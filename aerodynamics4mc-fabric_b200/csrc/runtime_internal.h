// Internal interface between the runtime translation units.
#pragma once

#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "d3q27_kernels.cuh"

namespace aero {

// Device state of one context (one brick / grid).
//
// g[cur] holds the post-collision populations of the last call. obstacle,
// ref_p and flags are double-buffered: index `slot` holds the inputs and pull
// classification of the last call, which the next call's fused kernel streams
// with (the reference streams at the end of each call with that call's mask).
// Bytes added after every per-cell array that the streamed in-place step
// reads with 16-byte-granular bulk copies (a run's last granule may extend
// up to 15 bytes past the array's last element).
constexpr size_t kCopySlack = 256;

struct Context {
    int nx = 0, ny = 0, nz = 0;
    long long cells = 0;
    int device = -1;  // CUDA device the context's memory lives on (current at allocation)
    float* g[2] = {nullptr, nullptr};
    uint8_t* obstacle[2] = {nullptr, nullptr};
    float* ref_p[2] = {nullptr, nullptr};
    uint32_t* flags[2] = {nullptr, nullptr};
    FaceParams* d_face[2] = {nullptr, nullptr};  // device copy of the faces each slot was classified with
    float* ref_ux = nullptr;
    float* ref_uy = nullptr;
    float* ref_uz = nullptr;
    float* temperature = nullptr;       // temperature the collision reads (transported state, or the packet field)
    float* temperature_next = nullptr;  // transport: the other state buffer
    float* temperature_scratch = nullptr;  // transport (BFECC): third state buffer
    float* ref_temperature = nullptr;   // transport: packet temperature channel
    float* thermal_source = nullptr;    // transport: packet source channel
    float* u_last = nullptr;            // transport: velocity of the last collision, SoA 3 x cells
    bool thermal = false;               // the current call runs the temperature transport
    float* packet = nullptr;
    size_t packet_cap = 0;
    float* out = nullptr;
    size_t out_cap = 0;
    float* force = nullptr;  // optional per-cell force density, SoA (3 * cells)
    int* fault = nullptr;    // device word: a streamed in-place step lost a tile's copies
    FaceParams face_prev{};
    FaceParams h_face[2]{};  // host copies (source of the async uploads; must outlive them)
    // Layout chosen at the first step: 0 two-buffer pull (g[0], g[1]),
    // 1 in-place esoteric pull (ip, padded by one ghost cell per side).
    int layout = 0;
    int ip_variant = 0;      // IpVariant when layout == 1
    void* ip = nullptr;      // padded population array (float or __half)
    float* solid_f = nullptr;
    // The face pre-fill a call leaves for the next one is deferred: the next
    // call's temperature update launches it in the same grid (independent
    // work), and anything else that touches the in-place populations first
    // launches it on the library stream (join_fill).
    bool fill_pending = false;
    cudaEvent_t copy_done = nullptr;  // a call's host-to-device input copies (returned only once read)
    float* fan_mask = nullptr;  // packet fan channels, 4 x cells (mask, ux, uy, uz), while fan forcing is on  // in-place: populations of solid cells (IpArgs::solid_f), from the first mask change on
    int parity = 0;          // slot-map parity of the next in-place step
    int periodic_mask = 0;   // axes wrapped by the in-place layout
    float fp16_scale = 0.0f; // per-brick FP16 deviation scale
    uint64_t bytes_per_step = 0;  // algorithmic population bytes per cell-step x cells
    void* scratch = nullptr; // conservation-sum partials
    size_t scratch_cap = 0;
    int cur = 0;
    // Two-buffer layout after a halo exchange: g[1 - cur] holds the streamed
    // state (exchanged slabs included); the next call collides it directly.
    bool f_ready = false;
    // compute_benchmark_force of the last call (cylinder preset): 3 device doubles
    double* force3 = nullptr;
    bool force_valid = false;
    // device copies of a call's sparse payload overlays
    int* overlay_cells = nullptr;
    float* overlay_values = nullptr;
    int overlay_cap = 0;
    // Block edits staged for the next call (its mask and classification in
    // this slot), or -1.
    int pending_slot = -1;
    int* patch_cells = nullptr;
    uint8_t* patch_solid = nullptr;
    int patch_cap = 0;
    // Boundary-reference shell (in-place): cells, layers, relaxation.
    void* shell = nullptr;
    int shell_count = 0;
    int shell_layers = 0;
    float shell_relax = 0.0f;
    int slot = 0;
    bool allocated = false;
    bool initialized = false;
    bool has_inputs = false;
    uint64_t step_counter = 0;

    Context() = default;
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    ~Context();
    bool allocate(int nx, int ny, int nz);
    void release_device();
    CellFields fields(int s) const;
    ForceField force_field() const;
};

struct RuntimeView {
    bool initialized;
    int nx, ny, nz;
    int input_channels, output_channels;
};

std::recursive_mutex& runtime_mutex();
void set_error(const std::string& msg);
void clear_error();
const std::string& last_error();
cudaStream_t current_stream();
bool cuda_ok(cudaError_t e, const char* what);
CollideParams current_collide_params();
FaceParams current_face_params();
int streaming_mode_setting();
int realtime_solver_mode();

Context* find_context(long long key);
Context* get_or_create_context(long long key, int nx, int ny, int nz);
void release_all_contexts();
const RuntimeView runtime_view();
// Sparse payload overlays of one call (host arrays; 6 values per cell).
struct SparseOverlays {
    const int* cells;
    const float* values;
    int count;
};
// One call of a context. packet: the call's input packet (host or device
// memory, host_packet saying which), or null for a cached call; fill (optional)
// builds the call's inputs on the device instead of a packet.
bool step_context(Context& ctx, const float* packet, float* out, float scale, bool host_packet,
                  const SparseOverlays* overlays = nullptr, const DeviceFill* fill = nullptr);
// aero_lbm_step_rect for a call whose inputs `fill` builds on the device:
// the same context lookup / creation, checks and timing record; no output.
bool step_rect_device(long long key, int nx, int ny, int nz, const DeviceFill& fill);
bool read_output(Context& ctx, int stride, int out_ch, float scale, float* host_out);
// Per-brick FP16 deviation scale for a brick whose speed stays below umax.
float fp16_scale_for_speed(float umax);
float i16_scale_for_speed(float umax);
// Device-side output into `dev_out` (no copy, no synchronisation).
bool output_device(Context& ctx, OutBox box, int out_ch, float scale, float* dev_out);
// Launches the face pre-fill the context's last call left pending (if any) on
// stream s, before anything on s reads the populations.
bool join_fill(Context& ctx, cudaStream_t s);
// Collect the slab copies of the following exchange_halo calls (in-place
// contexts) and launch them together at halo_batch_flush(); exchanges of one
// batch must touch disjoint slabs (the face slabs of a brick world do).
void halo_batch_begin();
bool halo_batch_flush();

}  // namespace aero
