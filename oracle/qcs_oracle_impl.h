/*
 * TEST INFRASTRUCTURE ONLY -- fixed-schedule MLEbfgs fit engine of the oracle.
 *
 * Included twice by qcs_oracle.c: REAL=float (suffix _f32) and REAL=double
 * (suffix _f64).  C_(x) spells a literal in REAL (0.1f in the float build).
 * Every arithmetic expression keeps the reference's operand order, so the
 * float build matches the reference bit for bit when both are compiled with
 * -ffp-contract=off against the same libm.
 *
 * Reference files (QC-STORM, MLEbfgs/bfgs_MLE_dll x64/bfgsMLE_dll/bfgsMLE_dll/):
 *   bfgsMLE_Loc_LD/bfgsMLE_core.h            scaling 52-60, BFGS helpers 65-238
 *   bfgsMLE_Loc_LD/bfgsMLE_GS2D_core.h       kernel 57-310, schedule 313-426,
 *                                            gradient 430-454, loss 459-518, pre-estimate 522-575
 *   bfgsMLE_Loc_LD/bfgsMLE_AS3D_core.h       kernel 58-337, loss 485-544, pre-estimate 548-607
 *   bfgsMLE_Loc_HD/bfgsMLE_GS2D_2Emitter_core.h  kernel 75-371, loss 519-592, pre-estimate 596-698
 *   bfgsMLE_Loc_HD/bfgsMLE_GS2D_3Emitter_core.h  kernel 77-362, loss 511-589, pre-estimate 593-710
 *   bfgsMLE_Loc_HD/bfgsMLE_AS3D_2Emitter_core.h  kernel 78-422, loss 570-644, pre-estimate 648-750
 */

#define FN_(a, b) a##b
#define FN2_(a, b) FN_(a, b)
#define FN(name) FN2_(name, SFX)

#if REAL_IS_DOUBLE
#define EXP_ exp
#define LOG_ log
#define SQRT_ sqrt
#define POW_ pow
#define MIN_ fmin
#define MAX_ fmax
#define C_(x) x
#else
#define EXP_ expf
#define LOG_ logf
#define SQRT_ sqrtf
#define POW_ powf
#define MIN_ fminf
#define MAX_ fmaxf
#define C_(x) x##f
#endif

/* Loss of one parameter vector.  The reference clamps the vector it is given
 * in place before evaluating (GS2D/2E/3E at 0, AS3D/AS3D-2E at 0.01), and the
 * caller keeps using the clamped values: the gradient and line search rely on
 * that, so q is written back. */
static REAL FN(loss)(int kind, int R, const REAL *img, const REAL *w, REAL *q)
{
    const struct qcso_kind *K = &KINDS[kind];
    const REAL lo = K->clamp_001 ? C_(0.01) : C_(0.0);
    for (int k = 0; k < K->npar; ++k)
        if (q[k] < lo) q[k] = lo;
    REAL total = C_(0.0);
    for (int row = 0; row < R; ++row) {
        const REAL rp = (REAL)row + C_(0.5);
        for (int col = 0; col < R; ++col) {
            const REAL cp = (REAL)col + C_(0.5);
            const REAL n = img[row * R + col];
            REAL mu;
            switch (kind) {
            case KIND_GS2D: {
                REAL dx = cp - q[1], dy = rp - q[2];
                REAL t = ((-(dx * dx + dy * dy)) * q[3]) * C_(0.1);
                mu = ((q[0] * C_(128.0)) * EXP_(t)) + (q[4] * C_(64.0));
                break;
            }
            case KIND_AS3D: {
                REAL dx = cp - q[1], dy = rp - q[2];
                REAL t = -((((dx * dx) * q[3]) * C_(0.1)) + (((dy * dy) * q[4]) * C_(0.1)));
                mu = ((q[0] * C_(128.0)) * EXP_(t)) + (q[5] * C_(64.0));
                break;
            }
            case KIND_2E: {
                REAL dx0 = cp - q[1], dy0 = rp - q[2];
                REAL dx1 = cp - q[4], dy1 = rp - q[5];
                REAL m0 = (q[0] * C_(128.0)) * EXP_(((-(dx0 * dx0 + dy0 * dy0)) * q[6]) * C_(0.1));
                REAL m1 = (q[3] * C_(128.0)) * EXP_(((-(dx1 * dx1 + dy1 * dy1)) * q[6]) * C_(0.1));
                mu = (m0 + m1) + (q[7] * C_(64.0));
                break;
            }
            case KIND_3E: {
                REAL dx0 = cp - q[1], dy0 = rp - q[2];
                REAL dx1 = cp - q[4], dy1 = rp - q[5];
                REAL dx2 = cp - q[7], dy2 = rp - q[8];
                REAL m0 = (q[0] * C_(128.0)) * EXP_(((-(dx0 * dx0 + dy0 * dy0)) * q[9]) * C_(0.1));
                REAL m1 = (q[3] * C_(128.0)) * EXP_(((-(dx1 * dx1 + dy1 * dy1)) * q[9]) * C_(0.1));
                REAL m2 = (q[6] * C_(128.0)) * EXP_(((-(dx2 * dx2 + dy2 * dy2)) * q[9]) * C_(0.1));
                mu = ((m0 + m1) + m2) + (q[10] * C_(64.0));
                break;
            }
            default: { /* KIND_AS3D2E */
                REAL dx0 = cp - q[1], dy0 = rp - q[2];
                REAL dx1 = cp - q[6], dy1 = rp - q[7];
                REAL m0 = (q[0] * C_(128.0)) *
                          EXP_(-((((dx0 * dx0) * q[3]) * C_(0.1)) + (((dy0 * dy0) * q[4]) * C_(0.1))));
                REAL m1 = (q[5] * C_(128.0)) *
                          EXP_(-((((dx1 * dx1) * q[8]) * C_(0.1)) + (((dy1 * dy1) * q[9]) * C_(0.1))));
                mu = (m0 + m1) + (q[10] * C_(64.0));
                break;
            }
            }
            const REAL dev = (mu - n) - n * (LOG_(mu) - LOG_(n));
            total = K->weighted ? total + w[row * R + col] * dev : total + dev;
        }
    }
    return total;
}

/* Central difference, +-0.002 in scaled units, one parameter after another on
 * a working copy that keeps the clamping of earlier evaluations. */
static void FN(numgrad)(int kind, int R, const REAL *img, const REAL *w, const REAL *x, REAL *g)
{
    const int P = KINDS[kind].npar;
    REAL t[QCSO_MAXPAR];
    for (int k = 0; k < P; ++k) t[k] = x[k];
    for (int k = 0; k < P; ++k) {
        t[k] = t[k] - C_(0.002);
        REAL ln = FN(loss)(kind, R, img, w, t);
        t[k] = t[k] + C_(0.004);
        REAL lp = FN(loss)(kind, R, img, w, t);
        g[k] = (lp - ln) * C_(250.0);
        t[k] = t[k] - C_(0.002);
    }
}

/* Rank-2 inverse-Hessian update D <- (I - s y'/y's) D (I - y s'/y's) + s s'/y's,
 * with the reference's summation order (bfgsMLE_core.h:88-182). */
static void FN(bfgs_update)(int P, REAL *D, const REAL *s, const REAL *y)
{
    REAL A[QCSO_MAXPAR * QCSO_MAXPAR], SS[QCSO_MAXPAR * QCSO_MAXPAR], T[QCSO_MAXPAR * QCSO_MAXPAR];
    REAL ya[QCSO_MAXPAR], sa[QCSO_MAXPAR];
    REAL sy = C_(0.0);
    for (int k = 0; k < P; ++k) sy += s[k] * y[k];
    sy = C_(1.0) / sy;
    for (int k = 0; k < P; ++k) {
        ya[k] = y[k] * sy;
        sa[k] = s[k] * sy;
    }
    for (int r = 0; r < P; ++r)
        for (int c = 0; c < P; ++c) {
            A[r * P + c] = (r == c ? C_(1.0) : C_(0.0)) - s[r] * ya[c];
            SS[r * P + c] = s[r] * sa[c];
        }
    for (int r = 0; r < P; ++r)
        for (int c = 0; c < P; ++c) {
            REAL acc = C_(0.0);
            for (int k = 0; k < P; ++k) acc += A[r * P + k] * D[k * P + c];
            T[r * P + c] = acc;
        }
    for (int r = 0; r < P; ++r)
        for (int c = 0; c < P; ++c) {
            REAL acc = C_(0.0);
            for (int k = 0; k < P; ++k) acc += T[r * P + k] * A[c * P + k];
            D[r * P + c] = acc;
        }
    for (int r = 0; r < P; ++r)
        for (int c = 0; c < P; ++c) D[r * P + c] = D[r * P + c] + SS[r * P + c];
}

/* The fixed schedule: IT iterations of a normalised quasi-Newton direction and
 * an 11-step bisection of the step length in [1e-5, 1]
 * (bfgsMLE_GS2D_core.h:313-426; identical in the other four fit kinds). */
static void FN(bfgs_fit)(int kind, int R, const REAL *img, const REAL *w, REAL *x)
{
    const struct qcso_kind *K = &KINDS[kind];
    const int P = K->npar, IT = K->iters, BS = 11;
    REAL D[QCSO_MAXPAR * QCSO_MAXPAR], g[QCSO_MAXPAR], d[QCSO_MAXPAR];
    REAL s[QCSO_MAXPAR], y[QCSO_MAXPAR], gold[QCSO_MAXPAR], xd[2][QCSO_MAXPAR];
    for (int r = 0; r < P; ++r)
        for (int c = 0; c < P; ++c) D[r * P + c] = (r == c) ? C_(1.0) : C_(0.0);
    FN(numgrad)(kind, R, img, w, x, g);
    for (int k = 0; k < P; ++k) d[k] = -g[k];
    for (int it = 0; it < IT; ++it) {
        REAL sum = C_(0.0);
        for (int k = 0; k < P; ++k) sum += FN(rabs)(d[k]);
        sum = ((REAL)P) / sum;
        for (int k = 0; k < P; ++k) d[k] = d[k] * sum;
        REAL lo = C_(0.00001), hi = C_(1.0);
        REAL dpos[2];
        dpos[0] = lo;
        dpos[1] = hi;
        REAL f[2];
        for (int k = 0; k < P; ++k) xd[0][k] = d[k] * C_(0.0001) + x[k];
        for (int k = 0; k < P; ++k) xd[1][k] = d[k] * C_(1.0) + x[k];
        f[0] = FN(loss)(kind, R, img, w, xd[0]);
        f[1] = FN(loss)(kind, R, img, w, xd[1]);
        for (int b = 0; b < BS; ++b) {
            const int sel = (f[0] < f[1]);
            dpos[sel] = (dpos[0] + dpos[1]) * C_(0.5);
            if (b < BS - 1) {
                for (int k = 0; k < P; ++k) xd[sel][k] = d[k] * dpos[sel] + x[k];
                f[sel] = FN(loss)(kind, R, img, w, xd[sel]);
            }
        }
        const REAL step = (dpos[0] + dpos[1]) * C_(0.5);
        for (int k = 0; k < P; ++k) {
            s[k] = d[k] * step;
            x[k] = x[k] + s[k];
        }
        for (int k = 0; k < P; ++k)
            if (x[k] < C_(0.01)) x[k] = C_(0.01);
        if (it < IT - 1) {
            for (int k = 0; k < P; ++k) gold[k] = g[k];
            FN(numgrad)(kind, R, img, w, x, g);
            for (int k = 0; k < P; ++k) y[k] = g[k] - gold[k];
            FN(bfgs_update)(P, D, s, y);
            for (int r = 0; r < P; ++r) {
                REAL acc = C_(0.0);
                for (int c = 0; c < P; ++c) acc -= D[r * P + c] * g[c];
                d[r] = acc;
            }
        }
    }
}

/* Gaussian weight mask of the weighted MLE (bfgsMLE_core.h:206-238). */
static void FN(wle_weights)(int R, REAL *w, REAL sx, REAL sy, int type)
{
    const REAL center = (REAL)R / C_(2.0);
    const REAL ax = C_(1.0) / ((C_(2.0) * sx) * sx);
    const REAL ay = C_(1.0) / ((C_(2.0) * sy) * sy);
    for (int row = 0; row < R; ++row)
        for (int col = 0; col < R; ++col) {
            const REAL rp = (REAL)row + C_(0.5), cp = (REAL)col + C_(0.5);
            if (type == QCS_MOLECULE_MLEFIT)
                w[row * R + col] = C_(1.0);
            else
                w[row * R + col] = EXP_(-((((cp - center) * (cp - center)) * ax) +
                                         (((rp - center) * (rp - center)) * ay)));
        }
}

/* Minimum of the edge-row / edge-column sums: shared by every pre-estimate. */
static void FN(edge_sums)(int R, const REAL *img, REAL *m1, REAL *m3)
{
    REAL a = C_(0.0), b = C_(0.0), c = C_(0.0), e = C_(0.0);
    for (int k = 0; k < R; ++k) {
        a += img[k * R + 0];
        b += img[k * R + R - 1];
        c += img[0 * R + k];
        e += img[(R - 1) * R + k];
    }
    *m1 = MIN_(a, b);
    *m3 = MIN_(c, e);
}

/* 3x3 block sums of a multi-emitter ROI; picks the brightest non-centre block
 * (and, for three emitters, the next one) as start positions. */
static void FN(block_starts)(int R, const REAL *img, int nstart, REAL *xs, REAL *ys)
{
    const int half = R / 2;
    const REAL center = (REAL)R / C_(2.0);
    const int len = R / 3 + 1, lenh = len / 2;
    int start[3] = {0, half - lenh, R - len};
    REAL pos[3] = {center - (REAL)len / C_(2.0), center, center + (REAL)len / C_(2.0)};
    REAL sums[9];
    for (int b = 0; b < 9; ++b) {
        REAL acc = C_(0.0);
        const int xb = start[b % 3], yb = start[b / 3];
        for (int r = 0; r < len; ++r)
            for (int c = 0; c < len; ++c) acc += img[(r + yb) * R + c + xb];
        sums[b] = acc;
    }
    sums[4] = C_(0.0);
    for (int e = 0; e < nstart; ++e) {
        int best = 0;
        for (int b = 0; b < 9; ++b)
            if (sums[b] > sums[best]) best = b;
        xs[e] = pos[best % 3];
        ys[e] = pos[best / 3];
        sums[best] = C_(0.0);
    }
}

/* Start vector of each fit kind (GS2D_core.h:522-575, AS3D_core.h:548-607,
 * 2Emitter_core.h:596-698, 3Emitter_core.h:593-710, AS3D_2Emitter_core.h:648-750). */
static void FN(pre_estimate)(int kind, int R, const REAL *img, REAL sx, REAL sy, REAL *x)
{
    const int half = R / 2;
    const REAL center = (REAL)R / C_(2.0);
    REAL m1, m3;
    FN(edge_sums)(R, img, &m1, &m3);
    if (kind == KIND_2E) {
        /* the two-emitter estimate takes the smaller edge mean alone */
        const REAL bkg = MIN_(m1, m3) / (REAL)R;
        const REAL amp = img[half * R + half] - bkg;
        const REAL s0 = (REAL)R / C_(2.2) / C_(2.35);
        const REAL s1 = C_(1.0) / ((C_(2.0) * s0) * s0);
        REAL xs[1], ys[1];
        FN(block_starts)(R, img, 1, xs, ys);
        x[0] = ((C_(0.8) * amp) * (C_(1.0) / (C_(128.0))));
        x[1] = center;
        x[2] = center;
        x[3] = ((C_(0.8) * amp) * (C_(1.0) / (C_(128.0))));
        x[4] = xs[0];
        x[5] = ys[0];
        x[6] = s1 * (C_(1.0) / (C_(0.1)));
        x[7] = ((C_(0.8) * bkg) * (C_(1.0) / (C_(64.0))));
        return;
    }
    const REAL bkg = ((m1 + m3) / (REAL)2) / (REAL)R;
    const REAL amp = img[half * R + half] - bkg;
    switch (kind) {
    case KIND_GS2D: {
        const REAL s1 = C_(1.0) / ((C_(2.0) * sx) * sx);
        x[0] = amp * (C_(1.0) / (C_(128.0)));
        x[1] = (REAL)half + C_(0.5);
        x[2] = (REAL)half + C_(0.5);
        x[3] = s1 * (C_(1.0) / (C_(0.1)));
        x[4] = bkg * (C_(1.0) / (C_(64.0)));
        break;
    }
    case KIND_AS3D: {
        x[0] = amp * (C_(1.0) / (C_(128.0)));
        x[1] = (REAL)half + C_(0.5);
        x[2] = (REAL)half + C_(0.5);
        x[3] = (C_(1.0) / (C_(0.1))) * (C_(0.5) / (sx * sx));
        x[4] = (C_(1.0) / (C_(0.1))) * (C_(0.5) / (sy * sy));
        x[5] = bkg * (C_(1.0) / (C_(64.0)));
        break;
    }
    case KIND_3E: {
        const REAL s0 = (REAL)R / C_(2.2) / C_(2.35);
        const REAL s1 = C_(1.0) / ((C_(2.0) * s0) * s0);
        REAL xs[2], ys[2];
        FN(block_starts)(R, img, 2, xs, ys);
        x[0] = ((C_(0.7) * amp) * (C_(1.0) / (C_(128.0))));
        x[1] = center;
        x[2] = center;
        x[3] = ((C_(0.7) * amp) * (C_(1.0) / (C_(128.0))));
        x[4] = xs[0];
        x[5] = ys[0];
        x[6] = ((C_(0.3) * amp) * (C_(1.0) / (C_(128.0))));
        x[7] = xs[1];
        x[8] = ys[1];
        x[9] = s1 * (C_(1.0) / (C_(0.1)));
        x[10] = ((C_(0.8) * bkg) * (C_(1.0) / (C_(64.0))));
        break;
    }
    default: { /* KIND_AS3D2E */
        const REAL s0 = (REAL)R / C_(2.2) / C_(2.35);
        const REAL s1 = (C_(1.0) / (C_(0.1))) * (C_(0.5) / (s0 * s0));
        REAL xs[1], ys[1];
        FN(block_starts)(R, img, 1, xs, ys);
        x[0] = ((C_(0.7) * amp) * (C_(1.0) / (C_(128.0))));
        x[1] = center;
        x[2] = center;
        x[3] = s1;
        x[4] = s1;
        x[5] = ((C_(0.7) * amp) * (C_(1.0) / (C_(128.0))));
        x[6] = xs[0];
        x[7] = ys[0];
        x[8] = s1;
        x[9] = s1;
        x[10] = ((C_(0.8) * bkg) * (C_(1.0) / (C_(64.0))));
        break;
    }
    }
}

/* Photoelectron image of one record: max((adu - Offset) * KAdc, 1). */
static void FN(load_roi)(const struct qcso_job *J, int id, REAL *img)
{
    const int R = J->R, whole = R * (R + 1);
    const uint16_t *rec = J->rois + (size_t)id * whole;
    for (int k = 0; k < R * R; ++k) {
#if REAL_IS_DOUBLE
        img[k] = MAX_(((REAL)rec[k] - (REAL)J->p->Offset) * (REAL)J->p->KAdc, C_(1.0));
#else
        img[k] = fmaxf(((float)rec[k] - J->p->Offset) * J->p->KAdc, 1.0f);
#endif
    }
}

static REAL FN(zpoly)(const qcs_loc_para *p, REAL d)
{
    REAL z;
    if (d >= C_(0.0))
        z = (REAL)p->p4_XGY * POW_(d, 4) + (REAL)p->p3_XGY * POW_(d, 3) + (REAL)p->p2_XGY * POW_(d, 2) +
            (REAL)p->p1_XGY * d + (REAL)p->p0_XGY;
    else
        z = (REAL)p->p4_XLY * POW_(d, 4) + (REAL)p->p3_XLY * POW_(d, 3) + (REAL)p->p2_XLY * POW_(d, 2) +
            (REAL)p->p1_XLY * d + (REAL)p->p0_XLY;
    return z * (REAL)p->ZDepthCorrFactor;
}

static void FN(header)(const struct qcso_job *J, int id, int *xo, int *yo, int *frame)
{
    const int R = J->R;
    const uint16_t *h = J->rois + (size_t)id * R * (R + 1) + R * R;
    *xo = h[0];
    *yo = h[1];
    *frame = h[2] + 65536 * h[3];
}

/* Single-emitter GS2D fit of record `id` (bfgsMLE_GS2D_core.h:170-308).
 * Returns 1 if accepted; otherwise *to2e says whether the multi-emitter
 * cascade takes the ROI (valid and SNR > 6). */
static int FN(fit_gs2d)(const struct qcso_job *J, int id, float *row, int *to2e)
{
    const int R = J->R, half = R / 2;
    const qcs_loc_para *p = J->p;
    REAL img[QCSO_MAXPIX], w[QCSO_MAXPIX], x[QCSO_MAXPAR];
    FN(load_roi)(J, id, img);
    int xo, yo, frame;
    FN(header)(J, id, &xo, &yo, &frame);
    const float *wle = J->wle + (size_t)id * QCS_WLE_PARA_NUM;
    const REAL cap = (REAL)R / C_(2.0) / C_(2.35);
    REAL sl = MIN_((REAL)wle[1], (REAL)wle[2]);
    REAL su = MIN_((REAL)wle[3], (REAL)wle[4]);
    const int type = (int)wle[5];
    REAL s = MIN_(sl, su);
    s = MIN_(s, cap);
    FN(pre_estimate)(KIND_GS2D, R, img, s, s, x);
    if (type != QCS_MOLECULE_MLEFIT) {
        s = s / C_(1.2);
        s = MIN_(s, cap);
    }
    if (p->WLEEn == 0 && type != QCS_MOLECULE_MULTIFIT) s = (REAL)R;
    FN(wle_weights)(R, w, s, s, type);
    FN(bfgs_fit)(KIND_GS2D, R, img, w, x);

    const REAL qe = (REAL)p->QE;
    const REAL peak = (x[0] * C_(128.0)) / qe;
    const REAL bkg = (x[4] * C_(64.0)) / qe;
    REAL fx = x[1], fy = x[2];
    REAL sig = x[3] * C_(0.1);
    sig = SQRT_(C_(0.5) / sig);
    if (isnan(fx)) fx = -1;
    if (isnan(fy)) fy = -1;
    if (isnan(sig)) sig = -1;
    const REAL snr = (SQRT_(qe) * peak) / SQRT_(peak + bkg);
    const REAL total = (((peak * (REAL)2) * C_(3.141593)) * sig) * sig;
    const REAL X = (fx - (REAL)half) + (REAL)xo;
    const REAL Y = (fy - (REAL)half) + (REAL)yo;
    const int valid = isnan(bkg) ? 0 : 1;
    const REAL smax = p->MultiEmitterFitEn ? (REAL)R / C_(2.0) / C_(2.35) : (REAL)R / C_(1.5) / C_(2.35);
    const REAL lb = (REAL)R / C_(2.0) - C_(1.5), ub = (REAL)R / C_(2.0) + C_(1.5);
    *to2e = 0;
    if (valid && snr > C_(4.0) && sig <= smax && sig >= C_(0.6) && fx > lb && fx < ub && fy > lb &&
        fy < ub) {
        row[QCS_POS_PPHO] = (float)peak;
        row[QCS_POS_XPOS] = (float)X;
        row[QCS_POS_YPOS] = (float)Y;
        row[QCS_POS_ZPOS] = 0.0f;
        row[QCS_POS_SIGX] = (float)sig;
        row[QCS_POS_SIGY] = (float)sig;
        row[QCS_POS_TPHO] = (float)total;
        row[QCS_POS_BAKG] = (float)bkg;
        row[QCS_POS_PSNR] = (float)snr;
        row[QCS_POS_FRME] = (float)frame;
        return 1;
    }
    if (p->MultiEmitterFitEn && valid && snr > C_(6.0)) *to2e = 1;
    for (int k = 0; k < QCS_OUT_PARA_NUM; ++k) row[k] = 0.0f;
    return 0;
}

/* Single-emitter astigmatic fit (bfgsMLE_AS3D_core.h:169-336). */
static int FN(fit_as3d)(const struct qcso_job *J, int id, float *row, int *to2e)
{
    const int R = J->R, half = R / 2;
    const qcs_loc_para *p = J->p;
    REAL img[QCSO_MAXPIX], w[QCSO_MAXPIX], x[QCSO_MAXPAR];
    FN(load_roi)(J, id, img);
    int xo, yo, frame;
    FN(header)(J, id, &xo, &yo, &frame);
    const float *wle = J->wle + (size_t)id * QCS_WLE_PARA_NUM;
    const int type = (int)wle[5];
    REAL sx = MIN_((REAL)wle[1], (REAL)wle[2]);
    REAL sy = MIN_((REAL)wle[3], (REAL)wle[4]);
    FN(pre_estimate)(KIND_AS3D, R, img, sx, sy, x);
    if (type != QCS_MOLECULE_MLEFIT) {
        const REAL cap = (REAL)R / C_(1.6) / C_(2.35);
        sx = MIN_(sx, cap);
        sy = MIN_(sy, cap);
    }
    if (p->WLEEn == 0 && type != QCS_MOLECULE_MULTIFIT) {
        sx = (REAL)R;
        sy = (REAL)R;
    }
    FN(wle_weights)(R, w, sx, sy, type);
    FN(bfgs_fit)(KIND_AS3D, R, img, w, x);

    const REAL qe = (REAL)p->QE;
    REAL peak = x[0] * C_(128.0);
    REAL bkg = x[5] * C_(64.0);
    REAL fx = x[1], fy = x[2];
    REAL gx = x[3] * C_(0.1), gy = x[4] * C_(0.1);
    gx = SQRT_(C_(0.5) / gx);
    gy = SQRT_(C_(0.5) / gy);
    if (isnan(fx)) fx = -1;
    if (isnan(fy)) fy = -1;
    if (isnan(gx)) gx = -1;
    if (isnan(gy)) gy = -1;
    const REAL snr = peak / SQRT_(peak + bkg);
    peak = peak / qe;
    bkg = bkg / qe;
    const REAL total = (((peak * (REAL)2) * C_(3.141593)) * gx) * gy;
    const REAL dif = gx * gx - gy * gy;
    const REAL z = FN(zpoly)(p, dif);
    const REAL X = (fx - (REAL)half) + (REAL)xo;
    const REAL Y = (fy - (REAL)half) + (REAL)yo;
    const REAL mean = (gx + gy) / (REAL)2;
    const int valid = isnan(bkg) ? 0 : 1;
    const REAL smax = p->MultiEmitterFitEn ? (REAL)R / C_(2.0) / C_(2.35) : (REAL)R / C_(1.5) / C_(2.35);
    const REAL lb = (REAL)R / C_(2.0) - C_(2.5), ub = (REAL)R / C_(2.0) + C_(2.5);
    *to2e = 0;
    if (valid && snr > C_(3.5) && mean > C_(0.8) && mean < smax && fx > lb && fx < ub && fy > lb &&
        fy < ub) {
        row[QCS_POS_PPHO] = (float)peak;
        row[QCS_POS_XPOS] = (float)X;
        row[QCS_POS_YPOS] = (float)Y;
        row[QCS_POS_ZPOS] = (float)z;
        row[QCS_POS_SIGX] = (float)gx;
        row[QCS_POS_SIGY] = (float)gy;
        row[QCS_POS_TPHO] = (float)total;
        row[QCS_POS_BAKG] = (float)bkg;
        row[QCS_POS_PSNR] = (float)snr;
        row[QCS_POS_FRME] = (float)frame;
        return 1;
    }
    if (p->MultiEmitterFitEn && valid && snr > C_(6.0)) *to2e = 1;
    for (int k = 0; k < QCS_OUT_PARA_NUM; ++k) row[k] = 0.0f;
    return 0;
}

/* Emitter ranking of the multi-emitter kernels: peak x (R - distance from the
 * ROI centre), with off-ROI coordinates pushed to -100
 * (2Emitter_core.h:245-271, 3Emitter_core.h:247-280). */
static void FN(rank_emitters)(int R, int ne, int stride, const REAL *x, int *sel0, int *sel1)
{
    const int half = R / 2;
    const REAL center = (REAL)R / C_(2.0);
    REAL score[3];
    for (int e = 0; e < ne; ++e) {
        REAL pk = x[stride * e + 0], cx = x[stride * e + 1], cy = x[stride * e + 2];
        if (FN(rabs)(cx - center) >= (REAL)half) cx = -100;
        if (FN(rabs)(cy - center) >= (REAL)half) cy = -100;
        REAL dist = SQRT_((cx - center) * (cx - center) + (cy - center) * (cy - center));
        score[e] = pk * ((REAL)R - dist);
    }
    int a = 0;
    for (int e = 0; e < ne; ++e)
        if (score[e] > score[a]) a = e;
    *sel0 = a;
    if (ne == 2) {
        *sel1 = 1 - a;
        return;
    }
    score[a] = -100;
    int b = 0;
    for (int e = 0; e < ne; ++e)
        if (score[e] > score[b]) b = e;
    *sel1 = b;
}

/* Multi-emitter fit of record `id` (GS2D 2E / GS2D 3E / AS3D 2E).  Writes the
 * first emitter into *row when accepted and the second into *extra when it
 * qualifies.  Return: 0 rejected, 1 first only, 2 first and second.  For the
 * 2E kinds a rejection sends the ROI on (*next = 1: 3E queue for GS2D, or the
 * rejected count for AS3D). */
static int FN(fit_multi)(const struct qcso_job *J, int kind, int id, float *row, float *extra)
{
    const int R = J->R, half = R / 2;
    const qcs_loc_para *p = J->p;
    const REAL center = (REAL)R / C_(2.0);
    REAL img[QCSO_MAXPIX], w[QCSO_MAXPIX], x[QCSO_MAXPAR];
    FN(load_roi)(J, id, img);
    int xo, yo, frame;
    FN(header)(J, id, &xo, &yo, &frame);
    const float *wle = J->wle + (size_t)id * QCS_WLE_PARA_NUM;
    REAL nn = C_(1000.0);
    if (kind == KIND_2E) {
        REAL s = (REAL)R / C_(1.8) / C_(2.35);
        nn = (REAL)wle[0];
        FN(pre_estimate)(KIND_2E, R, img, s, s, x);
        if (p->WLEEn == 0) s = (REAL)R;
        FN(wle_weights)(R, w, s, s, QCS_MOLECULE_MULTIFIT);
    } else {
        FN(pre_estimate)(kind, R, img, C_(0.0), C_(0.0), x);
        for (int k = 0; k < R * R; ++k) w[k] = C_(1.0); /* unweighted kinds never read it */
    }
    FN(bfgs_fit)(kind, R, img, w, x);
    const REAL qe = (REAL)p->QE;

    if (kind == KIND_AS3D2E) {
        x[0] = (x[0] * C_(128.0)) / qe;
        x[5] = (x[5] * C_(128.0)) / qe;
        x[3] = SQRT_(C_(0.5) / (x[3] * C_(0.1)));
        x[4] = SQRT_(C_(0.5) / (x[4] * C_(0.1)));
        x[8] = SQRT_(C_(0.5) / (x[8] * C_(0.1)));
        x[9] = SQRT_(C_(0.5) / (x[9] * C_(0.1)));
        const REAL bkg = (x[10] * C_(64.0)) / qe;
        const int valid = isnan(bkg) ? 0 : 1;
        int a, b;
        FN(rank_emitters)(R, 2, 5, x, &a, &b);
        const REAL smax = (REAL)R / C_(1.9) / C_(2.35), smin = C_(0.8);
        REAL pk[2], ex[2], ey[2], gx[2], gy[2], tot[2], snr[2], z[2], mean[2];
        const int sel[2] = {a, b};
        for (int e = 0; e < 2; ++e) {
            const int o = 5 * sel[e];
            pk[e] = x[o];
            ex[e] = x[o + 1];
            ey[e] = x[o + 2];
            gx[e] = x[o + 3];
            gy[e] = x[o + 4];
            tot[e] = (((pk[e] * (REAL)2) * C_(3.141593)) * gx[e]) * gy[e];
            snr[e] = (SQRT_(qe) * pk[e]) / SQRT_(pk[e] + bkg);
            z[e] = FN(zpoly)(p, gx[e] * gx[e] - gy[e] * gy[e]);
            mean[e] = (gx[e] + gy[e]) / (REAL)2;
        }
        const REAL dist = SQRT_((ex[0] - ex[1]) * (ex[0] - ex[1]) + (ey[0] - ey[1]) * (ey[0] - ey[1]));
        if (valid && snr[0] > C_(5.5) && mean[0] > C_(0.6) && mean[0] > smin && mean[0] <= smax) {
            FN(write_row)(row, pk[0], (ex[0] - (REAL)half) + (REAL)xo, (ey[0] - (REAL)half) + (REAL)yo, z[0],
                          gx[0], gy[0], tot[0], bkg, snr[0], frame);
            if (dist > C_(1.5) && snr[1] > C_(5.2) && nn > center && mean[1] > C_(0.6) && mean[1] > smin &&
                mean[1] <= smax && pk[1] > pk[0] / C_(3.0) && ex[1] > (REAL)1 && ey[1] > (REAL)1 &&
                ex[1] < (REAL)(R - 1) && ey[1] < (REAL)(R - 1)) {
                FN(write_row)(extra, pk[1], (ex[1] - (REAL)half) + (REAL)xo, (ey[1] - (REAL)half) + (REAL)yo,
                              z[1], gx[1], gy[1], tot[1], bkg, snr[1], frame);
                return 2;
            }
            return 1;
        }
        for (int k = 0; k < QCS_OUT_PARA_NUM; ++k) row[k] = 0.0f;
        return 0;
    }

    /* GS2D two / three emitters: shared sigma and background */
    const int ne = (kind == KIND_3E) ? 3 : 2;
    const int is = (kind == KIND_3E) ? 9 : 6, ib = (kind == KIND_3E) ? 10 : 7;
    REAL bkg;
    if (kind == KIND_3E) {
        bkg = (x[ib] * C_(64.0)) / qe;
        for (int e = 0; e < 3; ++e) x[3 * e] = (x[3 * e] * C_(128.0)) / qe;
    } else {
        x[0] = (x[0] * C_(128.0)) / qe;
        x[3] = (x[3] * C_(128.0)) / qe;
        bkg = (x[ib] * C_(64.0)) / qe;
    }
    const REAL sig = SQRT_(C_(0.5) / (x[is] * C_(0.1)));
    const int valid = isnan(bkg) ? 0 : 1;
    int a, b;
    FN(rank_emitters)(R, ne, 3, x, &a, &b);
    const REAL smax = (REAL)R / C_(2.0) / C_(2.35);
    const REAL pk0 = x[3 * a], x0 = x[3 * a + 1], y0 = x[3 * a + 2];
    const REAL pk1 = x[3 * b], x1 = x[3 * b + 1], y1 = x[3 * b + 2];
    const REAL tot0 = (((pk0 * (REAL)2) * C_(3.141593)) * sig) * sig;
    const REAL tot1 = (((pk1 * (REAL)2) * C_(3.141593)) * sig) * sig;
    const REAL snr0 = (SQRT_(qe) * pk0) / SQRT_(pk0 + bkg);
    const REAL snr1 = (SQRT_(qe) * pk1) / SQRT_(pk1 + bkg);
    const REAL dist = SQRT_((x0 - x1) * (x0 - x1) + (y0 - y1) * (y0 - y1));
    if (valid && snr0 > C_(5.5) && sig > C_(0.6) && sig <= smax) {
        FN(write_row)(row, pk0, (x0 - (REAL)half) + (REAL)xo, (y0 - (REAL)half) + (REAL)yo, C_(0.0), sig, sig,
                      tot0, bkg, snr0, frame);
        const int nn_ok = (kind == KIND_3E) ? (nn > center) : (nn >= center);
        if (dist > C_(1.5) && snr1 > C_(5.2) && nn_ok && pk1 > pk0 / C_(2.0) && x1 > (REAL)1 &&
            y1 > (REAL)1 && x1 < (REAL)(R - 1) && y1 < (REAL)(R - 1)) {
            FN(write_row)(extra, pk1, (x1 - (REAL)half) + (REAL)xo, (y1 - (REAL)half) + (REAL)yo, C_(0.0), sig,
                          sig, tot1, bkg, snr1, frame);
            return 2;
        }
        return 1;
    }
    for (int k = 0; k < QCS_OUT_PARA_NUM; ++k) row[k] = 0.0f;
    return 0;
}

/* LDLocData_TypeDef::BFGS_MLELocalization (bfgs_top.cu:26-204): classify,
 * single-emitter fit, 2E (and for GS2D 3E) cascade, CRLB.  Queues are built
 * in ascending ROI order and second emitters are appended in queue order, the
 * order a one-block-at-a-time execution of the reference produces. */
static int FN(localize)(const qcs_loc_para *p, const uint16_t *rois, const float *wle, int n, float *out,
                        int out_cap, int *n_valid, float *ratios)
{
    struct qcso_job J = {p, rois, wle, p->ROISize};
    if (n_valid) *n_valid = 0;
    if (ratios)
        for (int k = 0; k < 7; ++k) ratios[k] = 0.0f;
    if (n <= 0) return QCS_OK;
    if (n > QCS_MAX_POINT_NUM) n = QCS_MAX_POINT_NUM;
    if (out_cap < n) return QCS_ERR_CAPACITY;
    const int multi = p->MultiEmitterFitEn;
    const int as3d = (p->LocType == QCS_LOCTYPE_AS3D);
    int *single = (int *)malloc(sizeof(int) * n);
    int *q2 = (int *)malloc(sizeof(int) * n);
    int *flag = (int *)malloc(sizeof(int) * n);
    int ns = 0, n2 = 0;
    for (int i = 0; i < n; ++i) {
        if (multi && (int)wle[(size_t)i * QCS_WLE_PARA_NUM + 5] > QCS_MOLECULE_WLEFIT)
            q2[n2++] = i;
        else
            single[ns++] = i;
    }
    const int n2_classify = n2;
    const float fdiv = (float)(n < 1 ? 1 : n);
    if (ratios) {
        ratios[0] = (float)ns / fdiv;
        ratios[3] = (float)ns / fdiv;
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int k = 0; k < ns; ++k) {
        const int id = single[k];
        int to2e = 0;
        if (as3d)
            FN(fit_as3d)(&J, id, out + (size_t)id * QCS_OUT_PARA_NUM, &to2e);
        else
            FN(fit_gs2d)(&J, id, out + (size_t)id * QCS_OUT_PARA_NUM, &to2e);
        flag[k] = to2e;
    }
    for (int k = 0; k < ns; ++k)
        if (flag[k]) q2[n2++] = single[k];
    int valid_rows = n;
    if (multi) {
        const int kind2 = as3d ? KIND_AS3D2E : KIND_2E;
        const int has2 = (p->LocType == QCS_LOCTYPE_GS2D) || as3d;
        float *extra = (float *)calloc((size_t)(n2 > 0 ? n2 : 1) * QCS_OUT_PARA_NUM, sizeof(float));
        int *res = (int *)malloc(sizeof(int) * (n2 > 0 ? n2 : 1));
        int n3 = 0, rejected = 0;
        int *q3 = (int *)malloc(sizeof(int) * (n2 > 0 ? n2 : 1));
        if (has2) {
#pragma omp parallel for schedule(dynamic, 16)
            for (int k = 0; k < n2; ++k)
                res[k] = FN(fit_multi)(&J, kind2, q2[k], out + (size_t)q2[k] * QCS_OUT_PARA_NUM,
                                       extra + (size_t)k * QCS_OUT_PARA_NUM);
            for (int k = 0; k < n2; ++k) {
                if (res[k] == 2 && valid_rows < out_cap && valid_rows < QCS_MAX_POINT_NUM) {
                    memcpy(out + (size_t)valid_rows * QCS_OUT_PARA_NUM, extra + (size_t)k * QCS_OUT_PARA_NUM,
                           sizeof(float) * QCS_OUT_PARA_NUM);
                    valid_rows++;
                } else if (res[k] == 2) {
                    valid_rows++;
                }
                if (res[k] == 0) {
                    if (as3d)
                        rejected++;
                    else
                        q3[n3++] = q2[k];
                }
            }
        }
        if (p->LocType == QCS_LOCTYPE_GS2D && n3 > 0) {
            float *extra3 = (float *)calloc((size_t)n3 * QCS_OUT_PARA_NUM, sizeof(float));
            int *res3 = (int *)malloc(sizeof(int) * n3);
#pragma omp parallel for schedule(dynamic, 16)
            for (int k = 0; k < n3; ++k)
                res3[k] = FN(fit_multi)(&J, KIND_3E, q3[k], out + (size_t)q3[k] * QCS_OUT_PARA_NUM,
                                        extra3 + (size_t)k * QCS_OUT_PARA_NUM);
            for (int k = 0; k < n3; ++k) {
                if (res3[k] == 2) {
                    if (valid_rows < out_cap && valid_rows < QCS_MAX_POINT_NUM)
                        memcpy(out + (size_t)valid_rows * QCS_OUT_PARA_NUM,
                               extra3 + (size_t)k * QCS_OUT_PARA_NUM, sizeof(float) * QCS_OUT_PARA_NUM);
                    valid_rows++;
                }
                if (res3[k] == 0) rejected++;
            }
            free(extra3);
            free(res3);
        }
        if (ratios) {
            ratios[1] = (float)n2 / fdiv;
            ratios[2] = (float)n3 / fdiv;
            ratios[3] = (float)(ns - (n2 - n2_classify)) / fdiv;
            if (p->LocType == QCS_LOCTYPE_GS2D) {
                ratios[4] = (float)(n2 - n3) / fdiv;
                ratios[5] = (float)(n3 - rejected) / fdiv;
            } else {
                ratios[4] = (float)(n2 - rejected) / fdiv;
            }
            ratios[6] = (float)rejected / fdiv;
        }
        free(extra);
        free(res);
        free(q3);
    }
    free(single);
    free(q2);
    free(flag);
    /* rows past the buffer are counted by the reference but never written */
    int rows = valid_rows < out_cap ? valid_rows : out_cap;
    if (rows > QCS_MAX_POINT_NUM) rows = QCS_MAX_POINT_NUM;
    qcso_crlb(p, out, rows);
    if (n_valid) *n_valid = rows;
    return QCS_OK;
}

/* Kernel-level single-emitter pass over every record (no cascade, no CRLB). */
static int FN(fit_single)(int kind, const qcs_loc_para *p, const uint16_t *rois, const float *wle, int n,
                          float *out)
{
    struct qcso_job J = {p, rois, wle, p->ROISize};
    qcs_loc_para q = *p;
    q.MultiEmitterFitEn = 0;
    J.p = &q;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        int to2e;
        if (kind == 1)
            FN(fit_as3d)(&J, i, out + (size_t)i * QCS_OUT_PARA_NUM, &to2e);
        else
            FN(fit_gs2d)(&J, i, out + (size_t)i * QCS_OUT_PARA_NUM, &to2e);
    }
    return QCS_OK;
}

#undef FN_
#undef FN2_
#undef FN
#undef EXP_
#undef LOG_
#undef SQRT_
#undef POW_
#undef MIN_
#undef MAX_
#undef C_
