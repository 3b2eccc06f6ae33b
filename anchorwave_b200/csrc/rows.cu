// Gapped alignment rows from KSW2 CIGARs on the device: the decoding AnchorWave's callers
// run on the host before the MAF writer (src/myImportandFunction/alignSlidingWindow.cpp:
// 307-324 and :855-875): M (and =, X) copies the next bases of both sequences, I copies the
// query and puts '-' in the reference row, D puts '-' in the query row and copies the
// reference.  One warp per pair walks its CIGAR; each operation's segment is written by
// the whole warp.
#include "aw_internal.h"
#include "../../include/anchorwave_b200.h"

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

namespace aw {
namespace {

struct RowPair {
    int64_t cig_off, q_off, t_off, row_off;
    int32_t n_cigar, pad;
};

__global__ void cigar_rows_kernel(const RowPair *pairs, int n, const uint32_t *cig, const char *qs, const char *ts,
                                  char *row_q, char *row_d) {
    const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const RowPair P = pairs[i];
    const uint32_t *c = cig + P.cig_off;
    const char *q = qs + P.q_off, *t = ts + P.t_off;
    char *rq = row_q + P.row_off, *rd = row_d + P.row_off;
    int64_t qp = 0, tp = 0, rp = 0;
    for (int k = 0; k < P.n_cigar; ++k) {
        const uint32_t w = c[k];
        const int64_t len = w >> 4;
        const uint32_t op = w & 0xf;
        const bool cq = op != 2, ct = op != 1;  // M/=/X consume both, I the query, D the reference
        for (int64_t x = lane; x < len; x += 32) {
            rq[rp + x] = cq ? q[qp + x] : '-';
            rd[rp + x] = ct ? t[tp + x] : '-';
        }
        if (cq) qp += len;
        if (ct) tp += len;
        rp += len;
    }
}

struct RowBuffers {
    DevBuf pairs, cig, qs, ts, rq, rd;
    std::vector<RowPair> hp;
    std::vector<uint32_t> hc;
    std::vector<char> hq, ht;
    cudaStream_t st = nullptr;
    ~RowBuffers() {
        pairs.release(), cig.release(), qs.release(), ts.release(), rq.release(), rd.release();
        if (st) cudaStreamDestroy(st);
    }
};

thread_local RowBuffers *tls_rows = nullptr;

}  // namespace
}  // namespace aw

using namespace aw;

extern "C" int aw_cigar_rows_batch(int n, const uint32_t *const *cigar, const int *n_cigar, const char *const *query,
                                   const int *qlen, const char *const *target, const int *tlen, char *row_q,
                                   char *row_d, int64_t *row_off, int *row_len, int64_t capacity) {
    if (n < 0 || (n > 0 && (!cigar || !n_cigar || !query || !qlen || !target || !tlen || !row_q || !row_d ||
                            !row_off || !row_len))) {
        set_error("aw_cigar_rows_batch: invalid arguments");
        return AW_E_INVAL;
    }
    if (n == 0) return AW_OK;
    if (!tls_rows) {
        tls_rows = new RowBuffers();
        static thread_local struct Reaper {
            ~Reaper() { delete tls_rows; tls_rows = nullptr; }
        } reaper;
        (void)reaper;
    }
    RowBuffers &R = *tls_rows;
    if (!R.st && cudaStreamCreateWithFlags(&R.st, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("aw_cigar_rows_batch: no CUDA stream");
        return AW_E_CUDA;
    }
    // layout and checks on the host: operation codes, and no operation running past the end
    // of its sequence (the reference asserts the CIGAR ends exactly at both ends)
    R.hp.resize(n);
    int64_t nc = 0, nq = 0, nt = 0, nr = 0;
    for (int i = 0; i < n; ++i) {
        if (n_cigar[i] < 0 || qlen[i] < 0 || tlen[i] < 0 || (n_cigar[i] > 0 && !cigar[i])) {
            set_error("aw_cigar_rows_batch: invalid pair");
            return AW_E_INVAL;
        }
        int64_t qa = 0, ta = 0, len = 0;
        for (int k = 0; k < n_cigar[i]; ++k) {
            const uint32_t op = cigar[i][k] & 0xf, l = cigar[i][k] >> 4;
            if (op == 0 || op == 7 || op == 8) qa += l, ta += l;
            else if (op == 1) qa += l;
            else if (op == 2) ta += l;
            else {
                set_error("aw_cigar_rows_batch: CIGAR operation other than M, I, D, =, X");
                return AW_E_INVAL;
            }
            len += l;
        }
        if (qa > qlen[i] || ta > tlen[i]) {
            set_error("aw_cigar_rows_batch: CIGAR consumes more than the sequence holds");
            return AW_E_INVAL;
        }
        RowPair &P = R.hp[i];
        P.cig_off = nc, P.q_off = nq, P.t_off = nt, P.row_off = nr, P.n_cigar = n_cigar[i], P.pad = 0;
        row_off[i] = nr;
        row_len[i] = (int)len;
        nc += n_cigar[i], nq += qlen[i], nt += tlen[i], nr += len;
    }
    if (nr > capacity) {
        set_error("aw_cigar_rows_batch: rows exceed the output capacity");
        return AW_E_INVAL;
    }
    R.hc.resize((size_t)nc + 1), R.hq.resize((size_t)nq + 1), R.ht.resize((size_t)nt + 1);
    for (int i = 0; i < n; ++i) {
        const RowPair &P = R.hp[i];
        if (n_cigar[i]) memcpy(R.hc.data() + P.cig_off, cigar[i], 4 * (size_t)n_cigar[i]);
        if (qlen[i]) memcpy(R.hq.data() + P.q_off, query[i], (size_t)qlen[i]);
        if (tlen[i]) memcpy(R.ht.data() + P.t_off, target[i], (size_t)tlen[i]);
    }
#define RCUDA(call)                                                                              \
    do {                                                                                         \
        const cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                                 \
            set_error((std::string("aw_cigar_rows_batch: ") + cudaGetErrorString(e_)).c_str()); \
            return AW_E_CUDA;                                                                    \
        }                                                                                        \
    } while (0)
    RCUDA(R.pairs.ensure(sizeof(RowPair) * (size_t)n));
    RCUDA(R.cig.ensure(4 * (size_t)nc + 16));
    RCUDA(R.qs.ensure((size_t)nq + 16));
    RCUDA(R.ts.ensure((size_t)nt + 16));
    RCUDA(R.rq.ensure((size_t)nr + 16));
    RCUDA(R.rd.ensure((size_t)nr + 16));
    RCUDA(cudaMemcpyAsync(R.pairs.p, R.hp.data(), sizeof(RowPair) * (size_t)n, cudaMemcpyHostToDevice, R.st));
    RCUDA(cudaMemcpyAsync(R.cig.p, R.hc.data(), 4 * (size_t)nc, cudaMemcpyHostToDevice, R.st));
    RCUDA(cudaMemcpyAsync(R.qs.p, R.hq.data(), (size_t)nq, cudaMemcpyHostToDevice, R.st));
    RCUDA(cudaMemcpyAsync(R.ts.p, R.ht.data(), (size_t)nt, cudaMemcpyHostToDevice, R.st));
    cigar_rows_kernel<<<(unsigned)((n + 7) / 8), 256, 0, R.st>>>(R.pairs.as<RowPair>(), n, R.cig.as<uint32_t>(),
                                                                 R.qs.as<char>(), R.ts.as<char>(), R.rq.as<char>(),
                                                                 R.rd.as<char>());
    RCUDA(cudaGetLastError());
    RCUDA(cudaMemcpyAsync(row_q, R.rq.p, (size_t)nr, cudaMemcpyDeviceToHost, R.st));
    RCUDA(cudaMemcpyAsync(row_d, R.rd.p, (size_t)nr, cudaMemcpyDeviceToHost, R.st));
    RCUDA(cudaStreamSynchronize(R.st));
#undef RCUDA
    return AW_OK;
}
