/*
 * TEST INFRASTRUCTURE ONLY -- post-localization stage of the CPU oracle.
 *
 * Restates ZeroLocalizationsRemovel_TypeDef::RemoveZeroLocalizations
 * (bfgsMLE_Loc_top/ZeroLocalizationsRemove.cu:21-186):
 *   without frame sorting: keep the rows whose peak photon count (column 0)
 *   exceeds 1.0, in row order (:64-102);
 *   with frame sorting: for each frame from first_frame to end_frame, keep the
 *   rows of that frame (column 11 truncated to int) whose peak photon count
 *   truncated to int exceeds 1 (:161-186), in row order within a frame (the
 *   order a one-thread-at-a-time run of the reference's atomics produces).
 */
#include <string.h>

#include "qcs_oracle.h"

static int trunc_i(float v)
{
    if (v != v) return 0;
    if (v >= 2147483647.0f) return 2147483647;
    if (v <= -2147483648.0f) return (-2147483647 - 1);
    return (int)v;
}

int qcso_zero_remove(const float *rows, int n, int sort_frame, int first_frame, int end_frame, float *out, int *n_out)
{
    if (!rows || !out || !n_out || n < 0) return QCS_ERR_ARG;
    int k = 0;
    if (!sort_frame) {
        for (int i = 0; i < n; ++i)
            if (rows[(size_t)i * 12 + 0] > 1.0f) memcpy(out + (size_t)k++ * 12, rows + (size_t)i * 12, 48);
    } else {
        for (int f = first_frame; f <= end_frame; ++f)
            for (int i = 0; i < n; ++i) {
                const float *r = rows + (size_t)i * 12;
                if ((float)trunc_i(r[0]) > 1.0f && trunc_i(r[11]) == f) memcpy(out + (size_t)k++ * 12, r, 48);
            }
    }
    *n_out = k;
    return QCS_OK;
}
