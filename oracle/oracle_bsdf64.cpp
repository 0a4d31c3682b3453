// TEST INFRASTRUCTURE ONLY -- the oracle's BSDF in double precision.
//
// oracle_bsdf.inc instantiated with R = double: the same formulas and
// operation order as the FP32 restatement the device follows, evaluated in
// double.  Tests compare it with the reference's own FP64 BSDF
// (integrators/megakernel/include/ReferenceBsdf.hpp) on the same queries: the
// two must agree to double rounding, so every FP32-vs-FP64 difference of the
// restatement is the rounding of FP32 arithmetic, not a different formula.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle64 {
namespace {

struct V3d {
    double x, y, z;
};
inline V3d operator+(V3d a, V3d b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3d operator-(V3d a, V3d b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3d operator-(V3d a) { return {-a.x, -a.y, -a.z}; }
inline V3d operator*(V3d a, V3d b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3d operator*(V3d a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3d operator*(double s, V3d a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3d operator/(V3d a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V3d a, V3d b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
inline V3d cross(V3d a, V3d b) {
    return {(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)};
}
inline bool finite3(V3d v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
inline bool nonneg3(V3d v) { return v.x >= 0.0 && v.y >= 0.0 && v.z >= 0.0; }
inline bool any_neg(V3d v) { return v.x < 0.0 || v.y < 0.0 || v.z < 0.0; }

using R = double;
using V = V3d;
inline V vv(R x, R y, R z) { return {x, y, z}; }
inline V spl(R s) { return {s, s, s}; }
inline R lcos(R x) { return std::cos(x); }
inline R lsin(R x) { return std::sin(x); }
#include "oracle_bsdf.inc"

V load3(const float* p) { return {double(p[0]), double(p[1]), double(p[2])}; }

}  // namespace
}  // namespace oracle64

extern "C" {

// oracle_bsdf_probe in double: 160-byte float queries (re_bsdf_query),
// results as the 32 doubles of the reference shim's ref_bsdf_probe.
void oracle_bsdf_probe64(const float* queries, uint32_t n, double* results) {
    using namespace oracle64;
    for (uint32_t i = 0; i < n; ++i) {
        const float* q = queries + size_t(i) * 40u;
        auto u32 = [&](int k) { uint32_t v; std::memcpy(&v, q + k, 4); return v; };
        const Ctx c{load3(q + 0), q[3], load3(q + 4), q[7], load3(q + 8), u32(11)};
        const Params p{load3(q + 12), q[15], load3(q + 16), q[19], load3(q + 20),
                       q[23], load3(q + 24), u32(27), u32(31), u32(35)};
        const V wo = load3(q + 28), wi = load3(q + 32), u = load3(q + 36);
        const Eval e = evaluate(c, p, wo, wi);
        const Smp sm = sample_bsdf(c, p, wo, u);
        double pdf_at = 0.0;
        if (sm.valid && !sm.delta) {
            const Eval e2 = evaluate(c, p, wo, sm.dir);
            pdf_at = (e2.valid && e2.measure == 1) ? e2.pdf : 0.0;
        }
        double* o = results + size_t(i) * 32u;
        auto put = [&](int k, V v, double w) { o[k] = v.x; o[k + 1] = v.y; o[k + 2] = v.z; o[k + 3] = w; };
        put(0, e.value, e.pdf);
        put(4, e.diff, double(e.measure));
        put(8, e.spec, double(e.lobe));
        put(12, sm.dir, sm.pdf);
        put(16, sm.value, sm.eta);
        put(20, sm.diff, double(sm.measure));
        put(24, sm.spec, double(sm.lobe));
        o[28] = e.valid ? 1.0 : 0.0;
        o[29] = sm.delta ? 1.0 : 0.0;
        o[30] = sm.valid ? 1.0 : 0.0;
        o[31] = pdf_at;
    }
}

}  // extern "C"
