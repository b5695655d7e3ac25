/* A plain C99 caller of the C ABI (include/xr.h, include/xr_learn.h): builds
 * a context from an xr_scan, reads it back, and checks the argument and
 * configuration errors that need no device.  Exit code 0 = every check held;
 * otherwise the number of the failed check. */
#include <stdio.h>
#include <string.h>

#include "xr.h"
#include "xr_learn.h"

int main(void) {
    const float rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    const float basis[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    const float zero3[3] = {0, 0, 0};
    xr_scan s;
    memset(&s, 0, sizeof(s));
    s.sdd = 1000.0f;
    s.sod = 500.0f;
    s.det_size = 2.0f;
    s.num_voxel = 8;
    s.num_detect = 12;
    s.num_proj = 4;
    s.num_cond = 1;
    s.num_basis = 3;
    s.rot = rot;
    s.trans = zero3;
    s.offset = zero3;
    s.basis = basis;
    xr_ctx *ctx = NULL;
    if (xr_create(&s, 0, &ctx) != XR_OK || !ctx) return 1;
    xr_scan back;
    if (xr_get_scan(ctx, &back) != XR_OK) return 2;
    if (back.num_voxel != 8 || back.num_detect != 12 || back.num_proj != 4 || back.num_basis != 3) return 3;
    if (xr_dev_forward_fiber(ctx, NULL, NULL, XR_ROTATE_CW) != XR_ERR_ARG) return 4;
    if (strlen(xr_last_error(ctx)) == 0) return 5;
    if (xr_dev_session_epoch(ctx, NULL) != XR_ERR_STATE) return 6;
    if (xr_set_option(ctx, XR_OPT_STORAGE, 1) != XR_OK) return 7;
    float dummy = 0.0f;
    if (xr_dev_forward_fiber(ctx, &dummy, &dummy, XR_ROTATE_CW) != XR_ERR_CONFIG) return 8;
    xr_destroy(ctx);
    s.num_voxel = 0;
    if (xr_create(&s, 0, &ctx) != XR_ERR_ARG) return 9;
    printf("%s\n", xr_version());
    return 0;
}
