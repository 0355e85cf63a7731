/* Rendering one frame through the C ABI from C or C++: create the scene
 * handle, render into host buffers, report errors with tpt_last_error().
 * tests/test_abi_layout.py compiles this file against the header. */
#include <stdio.h>

#include "tinypt_cuda.h"

/* desc: the flattened scene; acc: w*h*3 doubles, acc_w: w*h doubles */
int render_frame(const tpt_scene_desc* desc, double* acc, double* acc_w) {
    void* scene = NULL;
    if (tpt_scene_create(desc, &scene) != TPT_OK) {
        fprintf(stderr, "%s\n", tpt_last_error());
        return -1;
    }
    tpt_render_config cfg = {.width = 1920, .height = 1080, .spp = 256, .max_bounces = 16, .rr_start = 3,
                             .tile = 16, .adaptive_min_spp = 8, .adaptive_threshold = 0.02,
                             .morton_enabled = 1, .mode = TPT_MODE_WAVEFRONT_FP32, .seed = 1};
    tpt_stats st = {0};
    const int rc = tpt_render(scene, &cfg, acc, acc_w, &st);
    if (rc != TPT_OK) fprintf(stderr, "%s\n", tpt_last_error());
    tpt_scene_destroy(scene);
    return rc;
}
