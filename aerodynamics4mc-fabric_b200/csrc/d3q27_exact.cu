// Instantiation of the brick-step kernels with the reference-order collision.
// Built with --fmad=false (see build.py): no multiply-add contraction, so the
// collision and output round exactly like the reference CPU step.
#include "ip_launch.h"

namespace aero {

cudaError_t launch_init_collide_exact(BrickDims d, CellFields cur, ForceField force, CollideParams cp, float* g_out,
                                   cudaStream_t stream) {
    return launch_init_collide_t<true>(d, cur, force, cp, g_out, stream);
}

cudaError_t launch_step_ab_exact(BrickDims d, const float* g_in, float* g_out, const uint32_t* flags_prev,
                              const uint8_t* obstacle_prev, const float* ref_p_prev, const FaceParams* face_prev,
                              CellFields cur, ForceField force, CollideParams cp, cudaStream_t stream) {
    return launch_step_ab_t<true>(d, g_in, g_out, flags_prev, obstacle_prev, ref_p_prev, face_prev, cur, force, cp,
                                   stream);
}

cudaError_t launch_collide_ab_exact(BrickDims d, float* f_io, CellFields cur, ForceField force, CollideParams cp,
                                 cudaStream_t stream) {
    return launch_collide_ab_t<true>(d, f_io, cur, force, cp, stream);
}

cudaError_t launch_output_ab_exact(BrickDims d, const float* g, const uint32_t* flags, const uint8_t* obstacle,
                                const float* ref_p, const FaceParams* face, OutBox box, int out_channels,
                                float velocity_scale, float* out, cudaStream_t stream, int direct) {
    return launch_output_ab_t<true>(d, g, flags, obstacle, ref_p, face, box, out_channels, velocity_scale, out,
                                     stream, direct);
}


cudaError_t ip_init_f32_exact(float* f, const IpArgs& a, cudaStream_t s) { return IpLaunch<StoreF32, true>::init(f, a, s); }
cudaError_t ip_fill_f32_exact(float* f, const IpArgs& a, cudaStream_t s) { return IpLaunch<StoreF32, true>::face_fill(f, a, s); }
cudaError_t ip_step_f32_exact(float* f, const IpArgs& a, bool transitions, cudaStream_t s) {
    return IpLaunch<StoreF32, true>::step(f, a, transitions, s);
}
cudaError_t ip_output_f32_exact(const float* f, const IpArgs& a, OutBox box, int out_ch, float scale, float* out, cudaStream_t s) {
    return IpLaunch<StoreF32, true>::output(f, a, box, out_ch, scale, out, s);
}

}  // namespace aero
