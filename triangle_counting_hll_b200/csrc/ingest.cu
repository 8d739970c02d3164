// ingest.cu -- device parsing of whitespace-separated edge-list text.
//
// Reference semantics: src/graph.py:8-26 and experiment/exp_gpu.py:131-144 --
// each line is stripped; empty lines and lines whose first character is a
// comment character are skipped; lines with fewer than two tokens are
// skipped; otherwise the first two tokens are parsed as integers (Python
// int(): optional sign, decimal digits).  A token that is not an integer
// makes the reference raise ValueError; here it is counted in *n_bad and the
// line is dropped, and the caller raises.
//
// Pipeline: flag line starts (byte after '\n', and byte 0) -> CUB flagged
// select of their offsets -> (one stream synchronisation to read the line
// count) -> one thread per line parses its first two tokens -> CUB flagged
// select of the parsed pairs.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "common.cuh"

namespace tchll {

struct CommentSet {
    uint32_t bits[8];  // 256-bit membership of comment characters
};

__device__ __forceinline__ bool is_ws(uint8_t c) {
    return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f';
}

__global__ void line_flag_kernel(const uint8_t* __restrict__ text, int64_t n, uint8_t* flag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || text[i - 1] == '\n') ? 1 : 0;
}

// Parse one token at text[*p] (stops at whitespace / end); returns false when
// the token is not an integer.
__device__ __forceinline__ bool parse_int(const uint8_t* text, int64_t end, int64_t& p, int64_t& out) {
    bool neg = false;
    if (p < end && (text[p] == '+' || text[p] == '-')) {
        neg = text[p] == '-';
        ++p;
    }
    int64_t v = 0;
    int nd = 0;
    bool overflow = false;
    while (p < end && !is_ws(text[p])) {
        const uint8_t c = text[p];
        if (c < '0' || c > '9') return false;
        if (v > (INT64_MAX - 9) / 10) overflow = true;
        v = v * 10 + (c - '0');
        ++nd;
        ++p;
    }
    if (nd == 0 || overflow) return false;
    out = neg ? -v : v;
    return true;
}

__global__ void parse_lines_kernel(const uint8_t* __restrict__ text, int64_t n, const int32_t* __restrict__ starts,
                                   int64_t n_lines, CommentSet cs, int32_t* u, int32_t* v, uint8_t* ok,
                                   unsigned long long* n_bad) {
    unsigned long long bad = 0;
    for (int64_t li = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; li < n_lines;
         li += (int64_t)gridDim.x * blockDim.x) {
        int64_t p = starts[li];
        const int64_t end = (li + 1 < n_lines) ? starts[li + 1] : n;
        uint8_t good = 0;
        while (p < end && is_ws(text[p])) ++p;  // strip
        if (p < end) {
            const uint8_t c0 = text[p];
            const bool comment = (cs.bits[c0 >> 5] >> (c0 & 31)) & 1u;
            if (!comment) {
                int64_t t1s = p;
                while (p < end && !is_ws(text[p])) ++p;
                int64_t t1e = p;
                while (p < end && is_ws(text[p])) ++p;
                if (p < end) {  // second token exists
                    int64_t a = 0, b = 0, q = t1s;
                    const bool oka = parse_int(text, t1e, q, a);
                    q = p;
                    const bool okb = parse_int(text, end, q, b);
                    if (oka && okb && a >= INT32_MIN && a <= INT32_MAX && b >= INT32_MIN && b <= INT32_MAX) {
                        u[li] = (int32_t)a;
                        v[li] = (int32_t)b;
                        good = 1;
                    } else {
                        ++bad;
                    }
                }
            }
        }
        ok[li] = good;
    }
    if (bad) atomicAdd(n_bad, bad);
}

struct IngestWs {
    uint8_t* flag;
    int32_t* starts;
    int64_t* n_lines;
    int32_t* tu;
    int32_t* tv;
    uint8_t* ok;
    void* tmp;
    size_t tmp_bytes;
};

static bool carve_ingest(void* ws, size_t bytes, int64_t n, IngestWs& W, size_t* need) {
    const size_t N = (size_t)(n > 0 ? n : 1);
    size_t a = 0, b = 0;
    cub::DeviceSelect::Flagged(nullptr, a, thrust::counting_iterator<int32_t>(0), (uint8_t*)nullptr,
                               (int32_t*)nullptr, (int64_t*)nullptr, (int)N);
    cub::DeviceSelect::Flagged(nullptr, b, (int32_t*)nullptr, (uint8_t*)nullptr, (int32_t*)nullptr,
                               (int64_t*)nullptr, (int)N);
    Carve cv(ws, bytes);
    W.flag = cv.take<uint8_t>(N);
    W.starts = cv.take<int32_t>(N);
    W.n_lines = cv.take<int64_t>(2);
    W.tu = cv.take<int32_t>(N);
    W.tv = cv.take<int32_t>(N);
    W.ok = cv.take<uint8_t>(N);
    W.tmp_bytes = a > b ? a : b;
    W.tmp = cv.take<char>(W.tmp_bytes);
    if (need) *need = cv.off;
    return cv.ok();
}

}  // namespace tchll

using namespace tchll;

TCHLL_EXPORT int tchll_ingest_workspace_bytes(int64_t n_bytes, size_t* bytes) {
    TCHLL_ARG(bytes && n_bytes >= 0 && n_bytes < (int64_t)INT32_MAX, "text must be shorter than 2^31 bytes");
    IngestWs W;
    carve_ingest(nullptr, 0, n_bytes, W, bytes);
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_parse_edges(const uint8_t* text, int64_t n_bytes, const char* comment_chars, int32_t* out_u,
                                   int32_t* out_v, int64_t* n_out, int64_t* n_bad, void* workspace,
                                   size_t workspace_bytes, void* stream) {
    // Synchronises `stream` once (to read the number of lines).
    TCHLL_ARG(n_bytes >= 0 && n_bytes < (int64_t)INT32_MAX, "text must be shorter than 2^31 bytes");
    TCHLL_ARG(n_out && n_bad && (n_bytes == 0 || (text && out_u && out_v)), "null pointer");
    IngestWs W;
    size_t need = 0;
    if (!carve_ingest(workspace, workspace_bytes, n_bytes, W, &need) || !workspace) {
        set_error("workspace too small: need %zu bytes, have %zu", need, workspace_bytes);
        return TCHLL_EWORKSPACE;
    }
    CommentSet cs;
    memset(&cs, 0, sizeof(cs));
    if (comment_chars)
        for (const unsigned char* c = (const unsigned char*)comment_chars; *c; ++c) cs.bits[*c >> 5] |= 1u << (*c & 31);
    cudaStream_t st = (cudaStream_t)stream;
    TCHLL_CUDA(cudaMemsetAsync(n_out, 0, sizeof(int64_t), st));
    TCHLL_CUDA(cudaMemsetAsync(n_bad, 0, sizeof(int64_t), st));
    if (n_bytes == 0) return TCHLL_OK;
    int64_t g = (n_bytes + 255) / 256;
    if (g > (int64_t)sm_count() * 32) g = (int64_t)sm_count() * 32;
    line_flag_kernel<<<(int)g, 256, 0, st>>>(text, n_bytes, W.flag);
    TCHLL_CHECK_LAUNCH("line_flag_kernel");
    size_t tb = W.tmp_bytes;
    TCHLL_CUDA(cub::DeviceSelect::Flagged(W.tmp, tb, thrust::counting_iterator<int32_t>(0), W.flag, W.starts,
                                          W.n_lines, (int)n_bytes, st));
    count_launch();
    int64_t n_lines = 0;
    TCHLL_CUDA(cudaMemcpyAsync(&n_lines, W.n_lines, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TCHLL_CUDA(cudaStreamSynchronize(st));
    if (n_lines <= 0) return TCHLL_OK;
    int64_t gl = (n_lines + 255) / 256;
    if (gl > (int64_t)sm_count() * 32) gl = (int64_t)sm_count() * 32;
    parse_lines_kernel<<<(int)gl, 256, 0, st>>>(text, n_bytes, W.starts, n_lines, cs, W.tu, W.tv, W.ok,
                                               (unsigned long long*)n_bad);
    TCHLL_CHECK_LAUNCH("parse_lines_kernel");
    tb = W.tmp_bytes;
    TCHLL_CUDA(cub::DeviceSelect::Flagged(W.tmp, tb, W.tu, W.ok, out_u, n_out, (int)n_lines, st));
    count_launch();
    tb = W.tmp_bytes;
    TCHLL_CUDA(cub::DeviceSelect::Flagged(W.tmp, tb, W.tv, W.ok, out_v, W.n_lines + 1, (int)n_lines, st));
    count_launch();
    return TCHLL_OK;
}
