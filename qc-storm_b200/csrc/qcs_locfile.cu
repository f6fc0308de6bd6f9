// Localization file: rows appended as 12 float32 each, native (little-endian)
// byte order, no header -- what the reference's worker writes after every
// batch (LocFile.Write(WriteLocArry, WriteLocNum * OutParaNumGS2D *
// sizeof(float)), Plugin for ImageJ/QC-STORM_ CPPDLL/QC-STORM_ CPPDLL/
// OnlineLocalizationLD.cpp:284) and what its loader reads
// (utility/Output file load and postprocessing/py_LoadBinaryLocData.py:
// np.fromfile(path, dtype=np.float32).reshape(-1, 12)).
//
// Rows already on the device (a localization's or a zero-row removal's
// output, count in device memory) are copied on the caller's stream into one
// of two pinned staging buffers and appended by a host function that the
// stream runs after the copy: the caller never waits for the GPU, and a
// buffer is reused only after the append that read it has finished.
#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"
#include "qcs_error.h"

using qcs::fail;

namespace {

struct Stage {
    float *rows = nullptr;  // pinned, capacity x 12
    int *count = nullptr;   // pinned
    int max_n = 0;
    cudaEvent_t done = nullptr;  // after the host append that read this buffer
    struct qcs_locfile *owner = nullptr;
};

}  // namespace

struct qcs_locfile {
    FILE *f = nullptr;
    long long rows = 0;
    int capacity = 0;
    int next = 0;
    int write_error = 0;  // set by a host append that failed
    Stage stage[2];
};

namespace {

// Runs on a CUDA-internal host thread after the stage's copies: no CUDA calls.
void CUDART_CB append_stage(void *arg) {
    Stage *st = static_cast<Stage *>(arg);
    qcs_locfile *lf = st->owner;
    int n = *st->count;
    if (n < 0) n = 0;
    if (n > st->max_n) n = st->max_n;
    if (n > 0 && fwrite(st->rows, sizeof(float) * QCS_OUT_PARA_NUM, (size_t)n, lf->f) != (size_t)n)
        lf->write_error = 1;
    else
        lf->rows += n;
}

}  // namespace

extern "C" {

int qcs_locfile_close(qcs_locfile *lf) {
    if (!lf) return QCS_OK;
    int st = QCS_OK;
    for (Stage &s : lf->stage) {
        if (!s.done) continue;  // never used: no CUDA resources
        cudaEventSynchronize(s.done);
        cudaEventDestroy(s.done);
        cudaFreeHost(s.rows);
        cudaFreeHost(s.count);
    }
    if (lf->f && fclose(lf->f) != 0) st = fail(QCS_ERR_ARG, "closing the localization file failed");
    if (lf->write_error && !st) st = fail(QCS_ERR_ARG, "writing the localization file failed");
    delete lf;
    return st;
}

int qcs_locfile_open(const char *path, int append, int capacity, qcs_locfile **out) {
    if (!out || !path) return fail(QCS_ERR_ARG, "null argument");
    *out = nullptr;
    if (capacity <= 0) capacity = 2 * QCS_MAX_POINT_NUM;
    qcs_locfile *lf = new qcs_locfile();
    lf->capacity = capacity;
    lf->f = fopen(path, append ? "ab" : "wb");
    if (!lf->f) {
        delete lf;
        return fail(QCS_ERR_ARG, "cannot open the localization file");
    }
    if (append) {
        fseek(lf->f, 0, SEEK_END);
        lf->rows = ftell(lf->f) / (long long)(sizeof(float) * QCS_OUT_PARA_NUM);
    }
    *out = lf;
    return QCS_OK;
}

int qcs_locfile_write(qcs_locfile *lf, const float *h_rows, int n) {
    if (!lf) return fail(QCS_ERR_ARG, "null file");
    if (n < 0) return fail(QCS_ERR_ARG, "negative row count");
    if (n == 0) return QCS_OK;
    if (!h_rows) return fail(QCS_ERR_ARG, "null rows");
    // rows queued from the device go first
    for (Stage &s : lf->stage)
        if (s.done) QCS_CUDA(cudaEventSynchronize(s.done), "pending device rows");
    if (lf->write_error) return fail(QCS_ERR_ARG, "writing the localization file failed");
    if (fwrite(h_rows, sizeof(float) * QCS_OUT_PARA_NUM, (size_t)n, lf->f) != (size_t)n)
        return fail(QCS_ERR_ARG, "writing the localization file failed");
    lf->rows += n;
    return QCS_OK;
}

int qcs_locfile_write_device(qcs_locfile *lf, const float *d_rows, const int *d_n, int max_n, void *stream) {
    if (!lf) return fail(QCS_ERR_ARG, "null file");
    if (max_n < 0) return fail(QCS_ERR_ARG, "negative row count");
    if (max_n > lf->capacity) return fail(QCS_ERR_CAPACITY, "row count above the file's staging capacity");
    if (max_n == 0) return QCS_OK;
    if (!d_rows) return fail(QCS_ERR_ARG, "null rows");
    if (lf->write_error) return fail(QCS_ERR_ARG, "writing the localization file failed");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Stage &st = lf->stage[lf->next];
    lf->next ^= 1;
    if (!st.rows) {
        QCS_CUDA(cudaMallocHost((void **)&st.rows, (size_t)lf->capacity * QCS_OUT_PARA_NUM * sizeof(float)),
                 "staging buffer");
        QCS_CUDA(cudaMallocHost((void **)&st.count, sizeof(int)), "staging count");
        QCS_CUDA(cudaEventCreateWithFlags(&st.done, cudaEventDisableTiming), "staging event");
        st.owner = lf;
    } else {
        // the append that last read this buffer has finished
        QCS_CUDA(cudaEventSynchronize(st.done), "staging buffer reuse");
    }
    st.max_n = max_n;
    if (d_n)
        QCS_CUDA(cudaMemcpyAsync(st.count, d_n, sizeof(int), cudaMemcpyDeviceToHost, s), "copy row count");
    else
        *st.count = max_n;
    // every slot a call can fill; the append writes the first *count
    QCS_CUDA(cudaMemcpyAsync(st.rows, d_rows, (size_t)max_n * QCS_OUT_PARA_NUM * sizeof(float),
                             cudaMemcpyDeviceToHost, s),
             "copy rows");
    QCS_CUDA(cudaLaunchHostFunc(s, append_stage, &st), "append rows");
    QCS_CUDA(cudaEventRecord(st.done, s), "record append");
    return QCS_OK;
}

int qcs_locfile_flush(qcs_locfile *lf) {
    if (!lf) return fail(QCS_ERR_ARG, "null file");
    for (Stage &s : lf->stage)
        if (s.done) QCS_CUDA(cudaEventSynchronize(s.done), "pending device rows");
    if (fflush(lf->f) != 0 || lf->write_error) return fail(QCS_ERR_ARG, "writing the localization file failed");
    return QCS_OK;
}

long long qcs_locfile_rows(const qcs_locfile *lf) { return lf ? lf->rows : -1; }

}  // extern "C"
