// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// extern "C" shim over the reference's own SVGF code, compiled from the
// unmodified reference sources by oracle/Makefile into oracle/_ref/:
//   - SvgfReconstruction::Process / SelectOutput  reconstruction/src/Svgf.cpp:408, 754
//   - ComputeRmse / ComputePsnr                   reconstruction/src/Svgf.cpp:824-841
//   - ComputeMotionVector                         reconstruction/src/MotionVectors.cpp:37
// Records use the flat C layouts of include/re_b200.h.
#include <cstdint>
#include <cstring>
#include <exception>

#include "reconstruction/MotionVectors.hpp"
#include "reconstruction/Svgf.hpp"

namespace rr = rendering::reconstruction;

namespace {

struct GbPix {
    float depth;
    float n[3];
    float dalb[3];
    float salb[3];
    float epd;
    float motion[2];
    uint32_t mat, obj, flags;
};
struct Config {
    float rel_depth, abs_depth, normal_cos;
    uint32_t require_mat, require_obj;
    uint32_t max_history;
    float min_color_alpha, min_moments_alpha;
    uint32_t short_history, radius;
    float min_variance;
    uint32_t iterations;
    float phi_depth, phi_normal, phi_luminance;
    float min_albedo;
    uint32_t demod_specular;
};
struct Outputs {
    float* raw;
    float* temporal;
    float* atrous;
    float* svgf;
    uint32_t* history_length;
    float* moments;
    float* variance;
    uint32_t* accepted;
    uint32_t* reject;
};

rr::SvgfConfig to_reference(const Config& c) {
    rr::SvgfConfig r{};
    r.validation.relativeDepthThreshold = c.rel_depth;
    r.validation.absoluteDepthThreshold = c.abs_depth;
    r.validation.normalCosineThreshold = c.normal_cos;
    r.validation.requireMaterialId = c.require_mat != 0u;
    r.validation.requireObjectId = c.require_obj != 0u;
    r.temporal.maxHistoryLength = c.max_history;
    r.temporal.minimumColorAlpha = c.min_color_alpha;
    r.temporal.minimumMomentsAlpha = c.min_moments_alpha;
    r.variance.shortHistoryLength = c.short_history;
    r.variance.spatialRadius = c.radius;
    r.variance.minimumVariance = c.min_variance;
    r.atrous.iterationCount = c.iterations;
    r.atrous.phiDepth = c.phi_depth;
    r.atrous.phiNormal = c.phi_normal;
    r.atrous.phiLuminance = c.phi_luminance;
    r.minimumAlbedo = c.min_albedo;
    r.demodulateSpecular = c.demod_specular != 0u;
    return r;
}

rr::Image<rr::GBufferPixel> gbuffer_image(const GbPix* gb, uint32_t w, uint32_t h) {
    rr::Image<rr::GBufferPixel> img({w, h});
    for (size_t i = 0; i < img.Size(); ++i) {
        const GbPix& g = gb[i];
        rr::GBufferPixel& p = img[i];
        p.linearDepth = g.depth;
        p.worldNormal = {g.n[0], g.n[1], g.n[2]};
        p.diffuseAlbedo = {g.dalb[0], g.dalb[1], g.dalb[2]};
        p.specularAlbedo = {g.salb[0], g.salb[1], g.salb[2]};
        p.expectedPreviousLinearDepth = g.epd;
        p.motion = {g.motion[0], g.motion[1]};
        p.materialId = g.mat;
        p.objectId = g.obj;
        p.valid = (g.flags & 1u) != 0u;
        p.motionValid = (g.flags & 2u) != 0u;
    }
    return img;
}

void copy_signal(const rr::Image<rr::SignalPixel>& img, float* dst) {
    for (size_t i = 0; i < img.Size(); ++i) std::memcpy(dst + 6 * i, &img[i], 24);
}

struct Handle {
    rr::SvgfReconstruction rec;
    rr::ReconstructionFrame last{};
    bool has_last = false;
    Handle(uint32_t w, uint32_t h, uint32_t f, const rr::SvgfConfig& c) : rec({w, h}, f, c) {}
};

}  // namespace

extern "C" {

void* ref_svgf_create(uint32_t w, uint32_t h, uint32_t flights, const Config* cfg) {
    try {
        return new Handle(w, h, flights, to_reference(*cfg));
    } catch (const std::exception&) {
        return nullptr;
    }
}

void ref_svgf_destroy(void* h) { delete static_cast<Handle*>(h); }

int ref_svgf_set_config(void* h, const Config* cfg) {
    try {
        static_cast<Handle*>(h)->rec.SetConfig(to_reference(*cfg));
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

int ref_svgf_process(void* hp, const GbPix* gb, const float* raw, uint32_t w, uint32_t h, uint64_t frame,
                     uint32_t trigger, const Outputs* out) {
    auto* hd = static_cast<Handle*>(hp);
    try {
        const rr::Image<rr::GBufferPixel> g = gbuffer_image(gb, w, h);
        rr::Image<rr::SignalPixel> s({w, h});
        for (size_t i = 0; i < s.Size(); ++i) std::memcpy(&s[i], raw + 6 * i, 24);
        hd->last = hd->rec.Process({g, s, frame, static_cast<rr::ResetTrigger>(trigger)});
        hd->has_last = true;
    } catch (const std::exception&) {
        return 1;
    }
    const rr::ReconstructionFrame& f = hd->last;
    copy_signal(f.raw, out->raw);
    copy_signal(f.temporal, out->temporal);
    copy_signal(f.atrous, out->atrous);
    copy_signal(f.svgf, out->svgf);
    for (size_t i = 0; i < f.raw.Size(); ++i) {
        out->history_length[i] = f.historyLength[i];
        out->moments[2 * i] = f.moments[i].first;
        out->moments[2 * i + 1] = f.moments[i].second;
        out->variance[i] = f.variance[i];
        out->accepted[i] = f.acceptedHistory[i];
        out->reject[i] = static_cast<uint32_t>(f.rejectReasons[i]);
    }
    return 0;
}

// SelectOutput of the last processed frame; 3 floats per pixel.
int ref_svgf_select(void* hp, const GbPix* gb, uint32_t w, uint32_t h, uint32_t output, float* dst) {
    auto* hd = static_cast<Handle*>(hp);
    if (!hd->has_last) return 1;
    try {
        const rr::Image<rr::Float3> img =
            hd->rec.SelectOutput(hd->last, gbuffer_image(gb, w, h), static_cast<rr::ReconstructionOutput>(output));
        for (size_t i = 0; i < img.Size(); ++i) std::memcpy(dst + 3 * i, &img[i], 12);
    } catch (const std::exception&) {
        return 1;
    }
    return 0;
}

float ref_image_rmse(const float* a, const float* b, uint32_t w, uint32_t h) {
    rr::Image<rr::Float3> x({w, h}), y({w, h});
    std::memcpy(x.Pixels().data(), a, 12 * x.Size());
    std::memcpy(y.Pixels().data(), b, 12 * y.Size());
    return rr::ComputeRmse(x, y);
}

float ref_image_psnr(const float* a, const float* b, uint32_t w, uint32_t h, float peak) {
    rr::Image<rr::Float3> x({w, h}), y({w, h});
    std::memcpy(x.Pixels().data(), a, 12 * x.Size());
    std::memcpy(y.Pixels().data(), b, 12 * y.Size());
    return rr::ComputePsnr(x, y, peak);
}

// ComputeMotionVector for an object at rest (identity object transforms).
void ref_motion_vector(const float* position, const float* cur_view_proj, const float* prev_view_proj,
                       const float* prev_world_to_view, const float* cur_jitter, const float* prev_jitter,
                       float* out) {
    rr::MotionVectorInput in{};
    in.objectPosition = {position[0], position[1], position[2]};
    std::memcpy(in.currentViewProjection.values.data(), cur_view_proj, 64);
    std::memcpy(in.previousViewProjection.values.data(), prev_view_proj, 64);
    std::memcpy(in.previousWorldToView.values.data(), prev_world_to_view, 64);
    in.currentJitterUv = {cur_jitter[0], cur_jitter[1]};
    in.previousJitterUv = {prev_jitter[0], prev_jitter[1]};
    const rr::MotionVectorResult r = rr::ComputeMotionVector(in);
    out[0] = r.currentUv.x;
    out[1] = r.currentUv.y;
    out[2] = r.previousUv.x;
    out[3] = r.previousUv.y;
    out[4] = r.motion.x;
    out[5] = r.motion.y;
    out[6] = r.expectedPreviousLinearDepth;
    out[7] = r.valid ? 1.0F : 0.0F;
}

}  // extern "C"
