// Test harness: host restatement of the two slab tests of
// renderingengine_b200/csrc/traverse.cuh -- the exact one (the reference's
// arithmetic, slab_test_planes) and the conservative one-fma form of
// traversal modes 7 and 8 (make_slab_ray_c, slab_test_planes_c,
// widen_limit) -- with the device's roundings: IEEE round-to-nearest for the
// plain operations, the directed roundings of __fmaf_ru / __fadd_ru /
// __fadd_rd through the floating-point environment.  Compiled by
// tests/test_slab_conservative.py with g++ -frounding-math
// -ffp-contract=off.
#include <cfenv>
#include <cmath>
#include <cstdint>

namespace {

float fmax3(float a, float b, float c) { return std::fmax(std::fmax(a, b), c); }  // NaN-ignoring, as max.f32
float fmin3(float a, float b, float c) { return std::fmin(std::fmin(a, b), c); }

// Directed roundings: the operands are read through volatiles after the
// mode switch, so the operation cannot be scheduled before it.
float add_dir(float a, float b, int mode) {
    volatile float va = a, vb = b;
    std::fesetround(mode);
    volatile float r = va + vb;
    std::fesetround(FE_TONEAREST);
    return r;
}
float fma_dir(float a, float b, float c, int mode) {
    volatile float va = a, vb = b, vc = c;
    std::fesetround(mode);
    volatile float r = std::fmaf(va, vb, vc);
    std::fesetround(FE_TONEAREST);
    return r;
}
float mul_rn(float a, float b) {
    volatile float r = a * b;
    return r;
}
float sub_rn(float a, float b) {
    volatile float r = a - b;
    return r;
}

struct Ray {
    float o[3], d[3], tmin;
};

// slab_test_planes: entry / exit planes chosen by the sign of 1 / d.
bool exact_test(const Ray& r, const float lo[3], const float hi[3], float limit, float& near_out) {
    float n[3], f[3];
    for (int a = 0; a < 3; ++a) {
        const float inv = 1.0f / r.d[a];
        const bool neg = std::signbit(inv);
        n[a] = mul_rn(sub_rn(neg ? hi[a] : lo[a], r.o[a]), inv);
        f[a] = mul_rn(sub_rn(neg ? lo[a] : hi[a], r.o[a]), inv);
    }
    const float tn = fmax3(n[0], n[1], n[2]);
    const float tf = fmin3(f[0], f[1], f[2]);
    near_out = std::fmax(tn, r.tmin);
    return !(tf < tn) && tf > r.tmin && tn < limit;
}

float widen_limit(float limit) {
    return add_dir(fma_dir(std::fabs(limit), 0x1p-21f, limit, FE_UPWARD), 0x1p-126f, FE_UPWARD);
}

// slab_constants + slab_test_planes_c.
bool conservative_test(const Ray& r, const float lo[3], const float hi[3], float limit_c, float& near_out) {
    float n[3], f[3];
    for (int a = 0; a < 3; ++a) {
        const float inv = 1.0f / r.d[a];
        const bool neg = std::signbit(inv);
        const float oi = mul_rn(r.o[a], inv);
        const float m = fma_dir(std::fabs(oi), 0x1p-22f, 0x1p-126f, FE_UPWARD);
        const float on = add_dir(oi, m, FE_UPWARD);
        const float of = add_dir(oi, -m, FE_DOWNWARD);
        n[a] = std::fmaf(neg ? hi[a] : lo[a], inv, -on);
        f[a] = std::fmaf(neg ? lo[a] : hi[a], inv, -of);
    }
    const float tn = fmax3(n[0], n[1], n[2]);
    const float tf = fmin3(f[0], f[1], f[2]);
    const float tfw = fma_dir(std::fabs(tf), 0x1p-21f, tf, FE_UPWARD);
    near_out = std::fmax(tn, r.tmin);
    return tfw >= near_out && near_out < limit_c;
}

}  // namespace

extern "C" {

// Per case: rays (o, d, tmin: 7 floats), boxes (lo, hi: 6 floats), limits.
// Writes the exact and the conservative verdicts and near distances.
void slab_compare(const float* rays, const float* boxes, const float* limits, uint32_t n, uint8_t* exact_hit,
                  uint8_t* cons_hit, float* exact_near, float* cons_near) {
    for (uint32_t i = 0; i < n; ++i) {
        Ray r;
        const float* x = rays + 7 * i;
        for (int a = 0; a < 3; ++a) {
            r.o[a] = x[a];
            r.d[a] = x[3 + a];
        }
        r.tmin = x[6];
        const float* b = boxes + 6 * i;
        float en, cn;
        exact_hit[i] = exact_test(r, b, b + 3, limits[i], en) ? 1 : 0;
        cons_hit[i] = conservative_test(r, b, b + 3, widen_limit(limits[i]), cn) ? 1 : 0;
        exact_near[i] = en;
        cons_near[i] = cn;
    }
}

}  // extern "C"
