/*
 * TEST INFRASTRUCTURE ONLY -- consecutive-frame merging of the CPU oracle.
 *
 * Restates ConsecutiveFit_TypeDef::ConsecutiveFit_WeightedAvg
 * (ConsecutiveFit/ConsecutiveFit_top.cu:22-98) and its three kernels
 * (ConsecutiveFit/ConsecutiveFit.cu:18-220), one group after another on one
 * state, every CUDA thread run in turn (no kernel reads what another thread
 * of the same launch writes, so the order does not matter):
 *   - the rows of the previous group (as this state left them) and the new
 *     group's rows form one array of T rows;
 *   - link: each row's x, y and frame truncated to int; scanning from the
 *     first row of its 32-row block while the last row read is at most one
 *     frame later, the closest row of the next frame whose squared integer
 *     distance is below the threshold (ConsecFit_DistanceTh_nm / PixelSize,
 *     squared), the first such row on ties; it gets a forward link, the row a
 *     backward link to it (or -2);
 *   - merge: every row without a forward link walks its backward chain while
 *     the id is > 0, summing peak, total photons and background and averaging
 *     x, y, z, sigma_x, sigma_y weighted by 10 / CRLB_x; the row takes the
 *     sums and averages and SNR sqrt(QE) peak / sqrt(peak + background);
 *     chains that start in the new group count their length in the on-time
 *     histogram (10 bins);
 *   - remove: the other rows of each chain are zeroed;
 *   - CRLB of the previous group's rows (now final) recomputed, and, as the
 *     reference's launch has no bound check (LocPrecCalc_GaussianCRLB.cu:23-40,
 *     32-thread blocks), of the new group's rows up to the next multiple of 32;
 *   - output: the previous group's rows, the new group kept for the next call
 *     (or, on the last call, everything).
 * gpu_rounding = 1 spells the weighted sums as the fused multiply-adds nvcc
 * makes of them and truncates NaN / out-of-range floats to int as the GPU
 * does (NaN -> 0, saturated); 0 keeps the separate roundings and x86
 * truncation (INT_MIN) of the reference's host build.  The CRLB is the host
 * restatement's (qcso_crlb) either way.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "qcs_oracle.h"

#define CF_ONTIME_BINS 10

static int trunc_mode(float v, int gpu)
{
    if (gpu) {
        if (v != v) return 0;
        if (v >= 2147483647.0f) return 2147483647;
        if (v <= -2147483648.0f) return (-2147483647 - 1);
        return (int)v;
    }
    if (v != v || v >= 2147483648.0f || v < -2147483648.0f) return (-2147483647 - 1);
    return (int)v;
}

/* wrapping int arithmetic of the reference's (X1 - X2)^2 + (Y1 - Y2)^2 */
static int dist2_int(int x1, int y1, int x2, int y2)
{
    const unsigned dx = (unsigned)x1 - (unsigned)x2, dy = (unsigned)y1 - (unsigned)y2;
    return (int)(dx * dx + dy * dy);
}

int qcso_consec(const qcs_loc_para *p, const float *rows, const int *sizes, const int *is_end, int n_groups,
                int gpu_rounding, float *out, int *out_n, float *ontime)
{
    if (!p || !rows || !sizes || !is_end || !out || !out_n || !ontime || n_groups < 0) return QCS_ERR_ARG;
    float *last = NULL;
    int last_n = 0;
    size_t off = 0, oo = 0;
    const float th_px = p->ConsecFit_DistanceTh_nm / p->PixelSize;
    for (int g = 0; g < n_groups; ++g) {
        const int cur = sizes[g];
        if (cur < 0) {
            free(last);
            return QCS_ERR_ARG;
        }
        const int T = last_n + cur;
        float *w = (float *)malloc(sizeof(float) * 12 * (size_t)(T > 0 ? T : 1));
        int *fwd = (int *)calloc((size_t)(T > 0 ? T : 1), sizeof(int));
        int *bwd = (int *)calloc((size_t)(T > 0 ? T : 1), sizeof(int));
        if (last_n) memcpy(w, last, sizeof(float) * 12 * (size_t)last_n);
        memcpy(w + (size_t)last_n * 12, rows + off * 12, sizeof(float) * 12 * (size_t)cur);
        int hist[CF_ONTIME_BINS] = {0};
        int valid = 0;
        /* link (gpuFindConsecutiveMolecules) */
        for (int gid = 0; gid < T; ++gid) {
            const float *r1 = w + (size_t)gid * 12;
            const int X1 = trunc_mode(r1[1], gpu_rounding), Y1 = trunc_mode(r1[2], gpu_rounding);
            const int F1 = trunc_mode(r1[11], gpu_rounding);
            int F2 = 0, paired = 0, similar = 0;
            float th2 = th_px;
            th2 = th2 * th2;
            for (int cnt = gid - gid % 32; cnt < T && F2 <= F1 + 1; ++cnt) {
                const float *r2 = w + (size_t)cnt * 12;
                const int X2 = trunc_mode(r2[1], gpu_rounding), Y2 = trunc_mode(r2[2], gpu_rounding);
                F2 = trunc_mode(r2[11], gpu_rounding);
                const float d2 = (float)dist2_int(X1, Y1, X2, Y2);
                if (d2 < th2 && F2 - F1 == 1) {
                    paired = cnt;
                    similar++;
                    th2 = d2;
                }
            }
            if (similar > 0) {
                bwd[gid] = paired;
                fwd[paired] = 1;
            } else {
                bwd[gid] = -2;
            }
        }
        /* merge (gpuConsecutiveFit) */
        for (int gid = 0; gid < T; ++gid) {
            if (fwd[gid] != 0) continue;
            float wx = 0, wy = 0, wz = 0, wsx = 0, wsy = 0, sp = 0, st = 0, sb = 0, sprec = 0;
            int id = gid, num = 0;
            for (;;) {
                const float *r = w + (size_t)id * 12;
                const float prec = 10.0f / r[9];
                sp += r[0];
                st += r[6];
                sb += r[7];
                if (gpu_rounding) {
                    wx = fmaf(r[1], prec, wx);
                    wy = fmaf(r[2], prec, wy);
                    wz = fmaf(r[3], prec, wz);
                    wsx = fmaf(r[4], prec, wsx);
                    wsy = fmaf(r[5], prec, wsy);
                } else {
                    wx += r[1] * prec;
                    wy += r[2] * prec;
                    wz += r[3] * prec;
                    wsx += r[4] * prec;
                    wsy += r[5] * prec;
                }
                sprec += prec;
                id = bwd[id];
                num++;
                if (!(id > 0)) break;
            }
            wx /= sprec;
            wy /= sprec;
            wz /= sprec;
            wsx /= sprec;
            wsy /= sprec;
            const float snr = sqrtf(p->QE) * sp / sqrtf(sp + sb);
            float *h = w + (size_t)gid * 12;
            h[0] = sp;
            h[1] = wx;
            h[2] = wy;
            h[3] = wz;
            h[4] = wsx;
            h[5] = wsy;
            h[6] = st;
            h[7] = sb;
            h[8] = snr;
            if (gid >= last_n) {
                int on = num - 1;
                if (on < 0) on = 0;
                if (on > CF_ONTIME_BINS - 1) on = CF_ONTIME_BINS - 1;
                valid++;
                hist[on]++;
            }
        }
        /* remove (gpuRemoveConsecutiveFluo) */
        for (int gid = 0; gid < T; ++gid) {
            if (fwd[gid] != 0) continue;
            int next = bwd[gid];
            while (next > 0) {
                memset(w + (size_t)next * 12, 0, sizeof(float) * 12);
                next = bwd[next];
            }
        }
        if (valid <= 0) valid = 1;
        for (int c = 0; c < CF_ONTIME_BINS; ++c) ontime[(size_t)g * CF_ONTIME_BINS + c] = hist[c] * 1.0f / valid;
        /* the reference's CRLB launch has no bound check: its 32-thread blocks
         * recompute every row up to the next multiple of 32 (within the T rows) */
        {
            int nc = (last_n + 31) / 32 * 32;
            if (nc > T) nc = T;
            if (nc) qcso_crlb(p, w, nc);
        }
        int outn;
        if (!is_end[g]) {
            outn = last_n;
            float *nl = (float *)malloc(sizeof(float) * 12 * (size_t)(cur > 0 ? cur : 1));
            memcpy(nl, w + (size_t)last_n * 12, sizeof(float) * 12 * (size_t)cur);
            memcpy(out + oo * 12, w, sizeof(float) * 12 * (size_t)outn);
            free(last);
            last = nl;
            last_n = cur;
        } else {
            outn = T;
            memcpy(out + oo * 12, w, sizeof(float) * 12 * (size_t)outn);
            free(last);
            last = NULL;
            last_n = 0;
        }
        out_n[g] = outn;
        oo += (size_t)outn;
        off += (size_t)cur;
        free(w);
        free(fwd);
        free(bwd);
    }
    free(last);
    return QCS_OK;
}
