// screen.cu -- screened path entry points (not built yet: the plain path
// serves every request).
#include "hm_internal.cuh"
#include "screen.cuh"

namespace hm {

int screen_plan(uint64_t, uint32_t, uint32_t, int, int path, ScreenLayout &) {
    return set_error(HM_ERR_UNSUPPORTED, "screened path %d is not available in this build", path);
}

int screen_run(const ScreenRun &, const ScreenLayout &, char *, cudaStream_t) {
    return set_error(HM_ERR_UNSUPPORTED, "screened path is not available in this build");
}

}  // namespace hm

extern "C" int hm_autotune_path(uint64_t, uint32_t, uint32_t, int) { return HM_PATH_PLAIN; }
