// AAFL compressed column blocks: the replacement of CompressionGPU::decompressDataAAFLOnDevice
// (qikkDB/Compression/GPUCompression.cu:474-522), whose decoder is feathergpu's gpu_aafl_decompress_kernel
// (fl/aafl.cuh:62-97): one thread per lane of each 32-lane group of rows unpacks its values one by one.
//
// Here one warp decodes one group (grid-stride over groups): lane l reads its stream words (consecutive lanes,
// consecutive words, so every load is one coalesced line), extracts value i from word (i b) / W at bit (i b) % W
// (and the next word when the value straddles two), adds the offset back, and the warp stores 32 consecutive rows
// per value index.  The same unpacking, row by row, feeds the fused aggregation pass (kz_key in groupby_fast.cuh).
#include <algorithm>
#include <limits>
#include <type_traits>

#include "aafl.cuh"

namespace qdb {

namespace {

template <typename T>
T offset_of(T mn, T mx) {
    // The block's min, or 0 when max - min does not fit T (GPUCompression.cu:33-38); -min wraps as two's complement
    // does for lowest(T).
    using U = typename std::make_unsigned<T>::type;
    T off = mn;
    if (mn < 0 && mx > 0) {
        const T neg = static_cast<T>(U(0) - static_cast<U>(mn));
        if (std::numeric_limits<T>::max() - mx < neg) off = 0;
    }
    return off;
}

template <typename WT>
__global__ void __launch_bounds__(256) aafl_decode_kernel(const WT* __restrict__ words, int64_t words_len,
                                                          const uint64_t* __restrict__ pos,
                                                          const uint8_t* __restrict__ bits, WT off, int64_t rows,
                                                          int64_t groups, WT* __restrict__ out,
                                                          unsigned* __restrict__ err) {
    constexpr int W = sizeof(WT) * 8;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; g < groups; g += warps) {
        const int b = bits[g];
        const int64_t base = static_cast<int64_t>(pos[g]) + lane;
        const int64_t d0 = g * 32 * W + lane;
        bool bad = false;
        for (int i = 0; i < W; ++i) {
            const int64_t d = d0 + 32 * i;
            if (d >= rows) break;
            WT x = 0;
            if (b) {
                const int o = i * b;
                const int p = o % W;
                const int64_t i0 = base + 32 * (o / W);
                const bool two = p + b > W;
                if (i0 >= 0 && i0 + (two ? 32 : 0) < words_len) {
                    x = words[i0] >> p;
                    if (two) x |= words[i0 + 32] << (W - p);
                    if (b < W) x &= (WT(1) << b) - WT(1);
                } else {
                    bad = true;
                }
            }
            out[d] = static_cast<WT>(x + off);
        }
        if (bad) atomicExch(err, 1u);
    }
}

// Compression, pass 1: per group, the bits of its largest (value - offset) and the words it takes (the last, partial
// group as GPUCompression.cu sizes it).
template <typename WT>
__global__ void __launch_bounds__(256) aafl_bits_kernel(const WT* __restrict__ in, int64_t rows, int64_t groups, WT off,
                                                        uint8_t* __restrict__ bits, long long* __restrict__ space) {
    constexpr int W = sizeof(WT) * 8;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; g < groups; g += warps) {
        const int64_t d0 = g * 32 * W;
        WT mx = 0;
        for (int64_t d = d0 + lane; d < rows && d < d0 + 32 * W; d += 32) mx = max(mx, static_cast<WT>(in[d] - off));
        for (int o = 16; o > 0; o >>= 1) {
            const WT y = __shfl_xor_sync(0xffffffffu, mx, o);
            mx = y > mx ? y : mx;
        }
        if (lane == 0) {
            int b = 0;
            if constexpr (W == 64) b = mx ? 64 - __clzll(static_cast<long long>(mx)) : 0;
            else b = mx ? 32 - __clz(static_cast<int>(mx)) : 0;
            const int64_t rem = rows - d0;
            long long sp = static_cast<long long>(b) * 32;
            if (rem < 32 * W) sp = ((((rem + W - 1) / W) * b + 31) / 32) * 32;
            bits[g] = static_cast<uint8_t>(b);
            space[g] = sp;
        }
    }
}

// Compression, pass 2: lane l of group g packs its values into its stream words at pos[g] + l + 32 k.
template <typename WT>
__global__ void __launch_bounds__(256) aafl_pack_kernel(const WT* __restrict__ in, int64_t rows, int64_t groups, WT off,
                                                        const uint8_t* __restrict__ bits,
                                                        const long long* __restrict__ pos, WT* __restrict__ words) {
    constexpr int W = sizeof(WT) * 8;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; g < groups; g += warps) {
        const int b = bits[g];
        if (b == 0) continue;
        const int64_t base = pos[g] + lane;
        WT acc = 0;
        int fill = 0;  // bits of acc in use
        int64_t k = 0;
        for (int i = 0; i < W; ++i) {
            const int64_t d = g * 32 * W + lane + 32 * i;
            if (d >= rows) break;
            const WT x = static_cast<WT>(in[d] - off);
            acc |= x << fill;
            if (fill + b >= W) {
                words[base + 32 * k++] = acc;
                const int used = W - fill;
                acc = used < W ? static_cast<WT>(x >> used) : WT(0);
                fill = b - used;
            } else {
                fill += b;
            }
        }
        if (fill > 0) words[base + 32 * k] = acc;
    }
}

// Exclusive scan of m word counts into positions, one block; *total receives the sum.
__global__ void __launch_bounds__(1024) aafl_scan_kernel(const long long* __restrict__ space, int64_t m,
                                                         long long* __restrict__ pos, long long* __restrict__ total) {
    __shared__ long long part[1024];
    const int64_t per = (m + 1023) / 1024;
    const int64_t b = threadIdx.x * per;
    const int64_t e = min(m, b + per);
    long long sum = 0;
    for (int64_t i = b; i < e; ++i) sum += space[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        const long long y = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
        __syncthreads();
        part[threadIdx.x] += y;
        __syncthreads();
    }
    long long run = part[threadIdx.x] - sum;
    for (int64_t i = b; i < e; ++i) {
        pos[i] = run;
        run += space[i];
    }
    if (threadIdx.x == 1023) *total = part[1023];
}

}  // namespace

int32_t aafl_view(const qdb_aafl_col* c, AaflView* v, cudaStream_t s, int align) {
    if (!c || !v || !c->data) return fail(QDB_ERR_INVALID, "AAFL block: null block");
    if (c->type != QDB_INT32 && c->type != QDB_INT64 && c->type != QDB_FLOAT)
        return fail(QDB_ERR_INVALID, "AAFL block: type must be INT32, INT64 or FLOAT");
    const int ws = c->type == QDB_INT64 ? 8 : 4;
    if (c->rows < 0 || c->blocks != (c->rows + 31) / 32)
        return fail(QDB_ERR_INVALID, "AAFL block: blocks must be ceil(rows / 32)");
    const int64_t meta = 24 + 9 * c->blocks;
    if (c->elements * ws < meta) return fail(QDB_ERR_INVALID, "AAFL block: shorter than its metadata");
    if (reinterpret_cast<uintptr_t>(c->data) & 7u) return fail(QDB_ERR_INVALID, "AAFL block: data must be 8-byte aligned");
    const char* base = static_cast<const char*>(c->data);
    *v = AaflView();
    v->word_bytes = ws;
    v->rows = c->rows;
    v->groups = (c->rows + 32 * 8 * ws - 1) / (32 * 8 * ws);
    v->pos = reinterpret_cast<const uint64_t*>(base + 24);
    v->bits = reinterpret_cast<const uint8_t*>(base + 24 + 8 * c->blocks);
    v->words_len = (c->elements * ws - meta) / ws;
    const char* words = base + meta;
    if (reinterpret_cast<uintptr_t>(words) % static_cast<uintptr_t>(std::max(align, ws)) != 0 && v->words_len > 0) {
        int32_t rc = dev_alloc(&v->scratch, static_cast<size_t>(v->words_len) * ws, s);
        if (rc != QDB_OK) return rc;
        QDB_CUDA_TRY(cudaMemcpyAsync(v->scratch, words, static_cast<size_t>(v->words_len) * ws, cudaMemcpyDeviceToDevice, s));
        words = static_cast<const char*>(v->scratch);
    }
    v->words = words;
    if (c->type == QDB_INT64) {
        v->off = static_cast<uint64_t>(offset_of<int64_t>(c->min_bits, c->max_bits));
    } else {
        int32_t mn = static_cast<int32_t>(static_cast<uint32_t>(c->min_bits));
        int32_t mx = static_cast<int32_t>(static_cast<uint32_t>(c->max_bits));
        if (c->type == QDB_FLOAT && mn > mx) std::swap(mn, mx);  // negative floats' bit patterns order the other way
        v->off = static_cast<uint32_t>(offset_of<int32_t>(mn, mx));
    }
    return QDB_OK;
}

}  // namespace qdb

using namespace qdb;

extern "C" {

int32_t qdb_aafl_decompress(const qdb_aafl_col* col, void* out, void* stream) {
    cudaStream_t s = as_stream(stream);
    AaflView v;
    int32_t rc = aafl_view(col, &v, s);
    if (rc != QDB_OK) return rc;
    if (v.rows == 0) return QDB_OK;
    if (!out) {
        dev_free(v.scratch, s);
        return fail(QDB_ERR_INVALID, "qdb_aafl_decompress: null output");
    }
    unsigned* err = nullptr;
    rc = dev_alloc(reinterpret_cast<void**>(&err), 4, s);
    if (rc == QDB_OK) {
        cudaError_t e = cudaMemsetAsync(err, 0, 4, s);
        const unsigned grid = static_cast<unsigned>(
            std::max<int64_t>(1, std::min<int64_t>((v.groups + 7) / 8, int64_t(device_info().sm_count) * 8)));
        if (e == cudaSuccess) {
            if (v.word_bytes == 8)
                aafl_decode_kernel<unsigned long long><<<grid, 256, 0, s>>>(
                    static_cast<const unsigned long long*>(v.words), v.words_len, v.pos, v.bits, v.off, v.rows,
                    v.groups, static_cast<unsigned long long*>(out), err);
            else
                aafl_decode_kernel<unsigned int><<<grid, 256, 0, s>>>(
                    static_cast<const unsigned int*>(v.words), v.words_len, v.pos, v.bits,
                    static_cast<unsigned int>(v.off), v.rows, v.groups, static_cast<unsigned int*>(out), err);
            note_launch();
            e = cudaGetLastError();
        }
        unsigned h = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(e, "aafl_decode_kernel");
        else if (h) rc = fail(QDB_ERR_INVALID, "qdb_aafl_decompress: a group's words lie outside the block");
    }
    dev_free(err, s);
    dev_free(v.scratch, s);
    return rc;
}

int32_t qdb_aafl_compress(int32_t type, const void* in, int64_t rows, int64_t min_bits, int64_t max_bits,
                          void** out_block, int64_t* out_elements, void* stream) {
    if (!out_block || !out_elements || rows < 0 || (rows > 0 && !in))
        return fail(QDB_ERR_INVALID, "qdb_aafl_compress: bad arguments");
    *out_block = nullptr;
    *out_elements = 0;
    if (type != QDB_INT32 && type != QDB_INT64 && type != QDB_FLOAT)
        return fail(QDB_ERR_INVALID, "qdb_aafl_compress: type must be INT32, INT64 or FLOAT");
    if (rows == 0) return QDB_OK;
    cudaStream_t s = as_stream(stream);
    const int ws = type == QDB_INT64 ? 8 : 4;
    uint64_t off = 0;
    if (type == QDB_INT64) {
        off = static_cast<uint64_t>(offset_of<int64_t>(min_bits, max_bits));
    } else {
        int32_t mn = static_cast<int32_t>(static_cast<uint32_t>(min_bits));
        int32_t mx = static_cast<int32_t>(static_cast<uint32_t>(max_bits));
        if (type == QDB_FLOAT) {
            // A float block is compressed only when its values share one sign (GPUCompression.cu:205).
            float fmn, fmx;
            memcpy(&fmn, &mn, 4);
            memcpy(&fmx, &mx, 4);
            if (!((fmn >= 0 && fmx >= 0) || (fmn <= 0 && fmx <= 0))) return QDB_OK;
            if (mn > mx) std::swap(mn, mx);
        }
        off = static_cast<uint32_t>(offset_of<int32_t>(mn, mx));
    }
    const int W = ws * 8;
    const int64_t blocks = (rows + 31) / 32;
    const int64_t groups = (rows + 32 * W - 1) / (32 * W);
    uint8_t* bits = nullptr;
    long long *space = nullptr, *pos = nullptr, *tot = nullptr;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&bits), static_cast<size_t>(groups), s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&space), static_cast<size_t>(groups) * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&pos), static_cast<size_t>(groups) * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&tot), 8, s);
    const unsigned grid = static_cast<unsigned>(
        std::max<int64_t>(1, std::min<int64_t>((groups + 7) / 8, int64_t(device_info().sm_count) * 8)));
    long long total = 0;
    if (rc == QDB_OK) {
        if (ws == 8)
            aafl_bits_kernel<unsigned long long><<<grid, 256, 0, s>>>(static_cast<const unsigned long long*>(in), rows,
                                                                      groups, off, bits, space);
        else
            aafl_bits_kernel<unsigned int><<<grid, 256, 0, s>>>(static_cast<const unsigned int*>(in), rows, groups,
                                                                static_cast<unsigned int>(off), bits, space);
        aafl_scan_kernel<<<1, 1024, 0, s>>>(space, groups, pos, tot);
        note_launch(2);
        cudaError_t e = cudaMemcpyAsync(&total, tot, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(e, "aafl_bits_kernel");
    }
    // The block's length as GPUCompression.cu:91-94 counts it; compression that does not shrink the block is dropped.
    const int64_t total_bytes = total * ws + std::max<int64_t>(8 * blocks, ws) + std::max<int64_t>(blocks, ws) + 24;
    const int64_t elems = (total_bytes + ws - 1) / ws;
    char* blk = nullptr;
    if (rc == QDB_OK && elems < rows) {
        rc = dev_alloc(reinterpret_cast<void**>(&blk), static_cast<size_t>(elems) * ws, s);
        const int64_t meta = 24 + 9 * blocks;
        void* words = nullptr;
        const bool aligned = meta % ws == 0;
        if (rc == QDB_OK && !aligned && total > 0) rc = dev_alloc(&words, static_cast<size_t>(total) * ws, s);
        if (rc == QDB_OK) {
            const int64_t hdr[3] = {rows, elems, blocks};
            cudaError_t e = cudaMemsetAsync(blk, 0, static_cast<size_t>(elems) * ws, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(blk, hdr, 24, cudaMemcpyHostToDevice, s);
            // position ids (uint64) and bit lengths, then the packed words
            if (e == cudaSuccess) e = cudaMemcpyAsync(blk + 24, pos, static_cast<size_t>(groups) * 8, cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(blk + 24 + 8 * blocks, bits, static_cast<size_t>(groups), cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess && total > 0) {
                if (!aligned) e = cudaMemsetAsync(words, 0, static_cast<size_t>(total) * ws, s);
                void* dst = aligned ? static_cast<void*>(blk + meta) : words;
                if (e == cudaSuccess) {
                    if (ws == 8)
                        aafl_pack_kernel<unsigned long long><<<grid, 256, 0, s>>>(
                            static_cast<const unsigned long long*>(in), rows, groups, off, bits, pos,
                            static_cast<unsigned long long*>(dst));
                    else
                        aafl_pack_kernel<unsigned int><<<grid, 256, 0, s>>>(
                            static_cast<const unsigned int*>(in), rows, groups, static_cast<unsigned int>(off), bits, pos,
                            static_cast<unsigned int*>(dst));
                    note_launch();
                    e = cudaGetLastError();
                }
                if (e == cudaSuccess && !aligned)
                    e = cudaMemcpyAsync(blk + meta, words, static_cast<size_t>(total) * ws, cudaMemcpyDeviceToDevice, s);
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the header above lives on this frame
            if (e != cudaSuccess) rc = cuda_fail(e, "aafl_pack_kernel");
        }
        dev_free(words, s);
    }
    dev_free(bits, s);
    dev_free(space, s);
    dev_free(pos, s);
    dev_free(tot, s);
    if (rc != QDB_OK) {
        dev_free(blk, s);
        return rc;
    }
    if (blk) {
        *out_block = blk;
        *out_elements = elems;
    }
    return QDB_OK;
}

}  // extern "C"
