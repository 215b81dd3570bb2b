// emit.cu -- frame emission on the device: vaco's pic_to_frame / blit
// (crates/codec/vaco-codec-av1/src/decode.rs:3795-3891).  The filtered u16
// planes are packed into the caller's frame layout: one byte per sample at
// 8 bits, where a value above 255 becomes 0 (blit's
// u8::try_from(v).unwrap_or(0)), and a little-endian u16 per sample above 8
// bits.  Bytes of a row past the copied width are left as they are, as blit
// leaves them.
//
// The kernel is a pure stream (read each sample once, write it once): a
// thread moves one 8-sample chunk per step, as 16-byte loads and 8- or
// 16-byte stores when the rows are aligned, over a grid-stride loop that
// walks every plane's chunks in order.
#include "common.cuh"
#include "kernels.cuh"

namespace vaco {

namespace {

constexpr int kEmitThreads = 256;

struct EmitArgs {
    EmitPlane p[3];
    int count;
    int two_bytes;
    int vec;
    int chunks_per_row[3];
    unsigned cpr_recip[3];    // fast_div_recip(chunks_per_row)
    long long chunk_base[4];  // first chunk of each plane; chunk_base[count] = total
};

// Two samples of one 32-bit word as two bytes (above 255 -> 0).
__device__ __forceinline__ uint32_t pack_bytes(uint32_t w) {
    const uint32_t lo = w & 0xFFFFu, hi = w >> 16;
    return (lo > 255u ? 0u : lo) | ((hi > 255u ? 0u : hi) << 8);
}

__global__ void __launch_bounds__(kEmitThreads) emit_kernel(EmitArgs a) {
    const long long total = a.chunk_base[a.count];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int p = 0;
        while (p + 1 < a.count && i >= a.chunk_base[p + 1]) ++p;
        const EmitPlane& P = a.p[p];
        const unsigned j = (unsigned)(i - a.chunk_base[p]);  // < 2^31 (checked on the host)
        const int cpr = a.chunks_per_row[p];
        const int y = (int)fast_div(j, cpr, a.cpr_recip[p]), x = (int)(j - (unsigned)y * cpr) * 8;
        const uint16_t* s = P.src + (long)y * P.src_stride + x;
        uint8_t* d = P.dst + (long long)y * P.dst_stride;
        const int n = min(8, P.width - x);
        if (a.vec && n == 8) {
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(s));
            if (a.two_bytes) {
                *reinterpret_cast<uint4*>(d + 2 * x) = q;
            } else {
                const uint2 b = make_uint2(pack_bytes(q.x) | (pack_bytes(q.y) << 16),
                                           pack_bytes(q.z) | (pack_bytes(q.w) << 16));
                *reinterpret_cast<uint2*>(d + x) = b;
            }
        } else {
            for (int k = 0; k < n; ++k) {
                const int v = s[k];
                if (a.two_bytes) {
                    d[2 * (x + k)] = (uint8_t)(v & 0xFF);
                    d[2 * (x + k) + 1] = (uint8_t)(v >> 8);
                } else {
                    d[x + k] = v > 255 ? 0 : (uint8_t)v;
                }
            }
        }
    }
}

}  // namespace

cudaError_t launch_emit(const EmitPlane* planes, int count, int two_bytes, int sm_count, cudaStream_t stream) {
    EmitArgs a;
    a.count = count;
    a.two_bytes = two_bytes;
    a.vec = 1;
    long long total = 0;
    for (int k = 0; k < count; ++k) {
        const EmitPlane& P = planes[k];
        a.p[k] = P;
        a.chunks_per_row[k] = (P.width + 7) / 8;
        a.cpr_recip[k] = fast_div_recip((unsigned)(a.chunks_per_row[k] > 0 ? a.chunks_per_row[k] : 1));
        if ((long long)a.chunks_per_row[k] * P.height >= (1LL << 31)) return cudaErrorInvalidValue;
        a.chunk_base[k] = total;
        total += (long long)a.chunks_per_row[k] * P.height;
        const unsigned dst_align = two_bytes ? 16u : 8u;
        a.vec = a.vec && (reinterpret_cast<uintptr_t>(P.src) % 16 == 0) && (P.src_stride % 8 == 0) &&
                (reinterpret_cast<uintptr_t>(P.dst) % dst_align == 0) && (P.dst_stride % dst_align == 0);
    }
    a.chunk_base[count] = total;
    if (total == 0) return cudaSuccess;
    // Enough CTAs to fill every SM several times over; each walks the chunks
    // with a grid stride.
    const long long want = (total + kEmitThreads - 1) / kEmitThreads;
    const int grid = (int)(want < (long long)sm_count * 8 ? want : (long long)sm_count * 8);
    emit_kernel<<<grid, kEmitThreads, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace vaco
