// GPU LBVH build (Morton codes, radix sort, Karras hierarchy, bottom-up refit).
#include "runtime.h"

namespace re {

re_status build_lbvh_on_device(re_scene* sc, const re_canonical_triangle* tris) {
    (void)sc;
    (void)tris;
    return set_error(RE_UNSUPPORTED, "GPU LBVH build is not available in this build");
}

}  // namespace re
