/* TEST INFRASTRUCTURE ONLY -- ROI extraction stage of the CPU oracle. */
#include "qcs_oracle.h"

int qcso_extract(const qcs_loc_para *p, const uint16_t *frames, int n_frames, int batch, int start_frame,
                 uint16_t *rois_out, float *wle_out, int cap, int *n_roi, int *first_frame, int *end_frame)
{
    (void)p; (void)frames; (void)n_frames; (void)batch; (void)start_frame; (void)rois_out;
    (void)wle_out; (void)cap; (void)n_roi; (void)first_frame; (void)end_frame;
    return QCS_ERR_NOT_BUILT;
}
