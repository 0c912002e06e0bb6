// transfer_codec.cu -- the transfer cache's byte format and the cache hit:
// a transfer set as an index and packed chunks (TransferSetCodec,
// MapTools/Rad/Bounce/TransferSetCodec.cs:23-447), written from and read
// back into the bounce's device transfer lists.
//
// The layout of the bytes is the reference's (every field little-endian):
//   index   "TRF1", patch count, longest list, total, every patch's count
//           (TransferSetCodec.Index, :31-45);
//   chunks  the transfers patch after patch as (patch, weight bits), a new
//           chunk every max(1, max_chunk_bytes / 8) transfers
//           (Chunks / ChunksIterator / Copy, :51-96);
//   packed  the chunk's count n, then a zlib stream of 8n bytes: byte b of
//           each patch delta as plane b, byte b of each weight as plane
//           4 + b (Pack, :105-133; Unpack, :140-188).
// The deflate stream is zlib's level 1; the reference's runtime may deflate
// the same planes to other bytes, and either reads the other's.
//
// Where the work runs.  The planes are byte-scatter work over the whole
// set (8 bytes a transfer, read once and written once), so the device does
// it: putting the lists in patch order, the deltas and the shuffle on the
// way out; the unshuffle and the deltas' prefix sum on the way in (one
// wrapping inclusive scan over every chunk's deltas, each chunk's base
// subtracted, which is exact modulo 2^32).  Deflate and inflate are
// sequential per chunk and run on the host's threads, a chunk to a thread.

#include <cuda_runtime.h>
#include <zlib.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdint>
#include <cstring>
#include <vector>

#include "bounce.cuh"
#include "context.cuh"
#include "host_parallel.h"
#include "sync_wait.h"

namespace vrad {

namespace {

constexpr int64_t kTransferBytes = 8;
// .NET's Array.MaxLength: the reference's bound on a count or a total.
constexpr int64_t kArrayMaxLength = 0x7FFFFFC7;

inline void put_u32(uint8_t *p, uint32_t v) {
    for (int b = 0; b < 4; b++) p[b] = (uint8_t)(v >> (8 * b));
}
inline void put_i64(uint8_t *p, int64_t v) {
    for (int b = 0; b < 8; b++) p[b] = (uint8_t)((uint64_t)v >> (8 * b));
}
inline uint32_t get_u32(const uint8_t *p) {
    return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
}
inline int64_t get_i64(const uint8_t *p) {
    uint64_t v = 0;
    for (int b = 0; b < 8; b++) v |= (uint64_t)p[b] << (8 * b);
    return (int64_t)v;
}

// Transfers a chunk holds: Math.Clamp(maxChunkBytes / 8, 1, int.MaxValue / 8).
inline int64_t per_chunk(int64_t max_chunk_bytes) {
    return std::clamp<int64_t>(max_chunk_bytes / kTransferBytes, 1, INT32_MAX / kTransferBytes);
}

// A zlib stream (RFC 1950) of in[0..n) at level 1 into out; its size, or -1
// when cap is too small.
int64_t deflate_fast(const uint8_t *in, int64_t n, uint8_t *out, int64_t cap) {
    z_stream zs;
    std::memset(&zs, 0, sizeof zs);
    if (deflateInit(&zs, 1) != Z_OK) return -1;
    zs.next_in = const_cast<Bytef *>(in);
    zs.avail_in = (uInt)n;
    zs.next_out = out;
    zs.avail_out = (uInt)std::min<int64_t>(cap, UINT_MAX);
    const int rc = deflate(&zs, Z_FINISH);
    const int64_t written = (int64_t)zs.total_out;
    deflateEnd(&zs);
    return rc == Z_STREAM_END ? written : -1;
}

// Bytes deflate_fast may need for n bytes of input.
inline int64_t deflate_room(int64_t n) { return (int64_t)compressBound((uLong)n); }

// True when the zlib stream in[0..len) inflates to exactly `want` bytes
// (into out) and no more: Unpack's ReadExactly followed by ReadByte() == -1.
// A stream that holds fewer bytes, more bytes or bad data fails.
bool inflate_exact(const uint8_t *in, int64_t len, uint8_t *out, int64_t want) {
    if (len < 0 || len > (int64_t)UINT_MAX || want > (int64_t)UINT_MAX) return false;
    z_stream zs;
    std::memset(&zs, 0, sizeof zs);
    if (inflateInit(&zs) != Z_OK) return false;
    zs.next_in = const_cast<Bytef *>(in);
    zs.avail_in = (uInt)len;
    zs.next_out = out;
    zs.avail_out = (uInt)want;
    int rc = Z_OK;
    while (zs.avail_out > 0) {
        rc = inflate(&zs, Z_NO_FLUSH);
        if (rc != Z_OK) break;
    }
    bool ok = zs.avail_out == 0 && (rc == Z_OK || rc == Z_STREAM_END);
    if (ok && rc != Z_STREAM_END) {
        // Full: the stream must end here (or run out of input: the
        // reference's inflater reads a stream cut after its last byte of
        // data as ended).
        uint8_t extra = 0;
        zs.next_out = &extra;
        zs.avail_out = 1;
        rc = inflate(&zs, Z_NO_FLUSH);
        ok = zs.avail_out == 1 && (rc == Z_STREAM_END || rc == Z_BUF_ERROR || rc == Z_OK);
    }
    inflateEnd(&zs);
    return ok;
}

// Pack's planes of one raw chunk, on the host.
void shuffle_host(const uint8_t *chunk, int64_t n, uint8_t *planes) {
    uint32_t previous = 0;
    for (int64_t k = 0; k < n; k++) {
        const uint32_t patch = get_u32(chunk + k * kTransferBytes);
        const uint32_t weight = get_u32(chunk + k * kTransferBytes + 4);
        const uint32_t delta = patch - previous;
        previous = patch;
        for (int b = 0; b < 4; b++) {
            planes[b * n + k] = (uint8_t)(delta >> (8 * b));
            planes[(4 + b) * n + k] = (uint8_t)(weight >> (8 * b));
        }
    }
}

// Unpack's inverse of shuffle_host.
void unshuffle_host(const uint8_t *planes, int64_t n, uint8_t *chunk) {
    uint32_t previous = 0;
    for (int64_t k = 0; k < n; k++) {
        uint32_t delta = 0, weight = 0;
        for (int b = 0; b < 4; b++) {
            delta |= (uint32_t)planes[b * n + k] << (8 * b);
            weight |= (uint32_t)planes[(4 + b) * n + k] << (8 * b);
        }
        previous += delta;
        put_u32(chunk + k * kTransferBytes, previous);
        put_u32(chunk + k * kTransferBytes + 4, weight);
    }
}

// TransferSetCodec.TryReadIndex (:329-372): the index fits patch_count, its
// counts add up to its total and their longest is its max.
bool read_index(const uint8_t *index, int64_t len, int32_t patch_count, std::vector<int32_t> &counts,
                int32_t &max, int64_t &total) {
    if (!index || patch_count < 0 || len < 20 || get_u32(index) != VRAD_TRANSFER_MAGIC ||
        (int32_t)get_u32(index + 4) != patch_count || len != 20 + 4 * (int64_t)patch_count)
        return false;
    max = (int32_t)get_u32(index + 8);
    total = get_i64(index + 12);
    if (total < 0 || total > kArrayMaxLength) return false;
    counts.resize((size_t)patch_count);
    int64_t at = 0;
    int32_t longest = 0;
    for (int32_t p = 0; p < patch_count; p++) {
        const int32_t c = (int32_t)get_u32(index + 20 + 4 * (int64_t)p);
        if (c < 0) return false;
        counts[(size_t)p] = c;
        at += c;
        longest = std::max(longest, c);
    }
    return at == total && longest == max;
}

}  // namespace

// ---- Device kernels ---------------------------------------------------------

namespace {

constexpr int kCodecBlock = 256;

// Grid-stride launches: enough CTAs to fill the device a few times over.
unsigned codec_grid(int64_t n, int sms) {
    const int64_t want = (n + kCodecBlock - 1) / kCodecBlock;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 16));
}

// The lists between the bounce's receiver order (tr_off / tr, receiver r's
// list for patch recv[r]) and patch order (arena, patch p's list at
// poff[p]).  One warp per receiver; TO_PATCH picks the direction.
template <bool TO_PATCH>
__global__ void k_reorder_lists(int32_t nrecv, const int32_t *__restrict__ recv, const int64_t *__restrict__ tr_off,
                                const int64_t *__restrict__ poff, int2 *__restrict__ tr, int2 *__restrict__ arena) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nrecv) return;
    const int64_t a = tr_off[warp], n = tr_off[warp + 1] - a, d = poff[recv[warp]];
    for (int64_t k = lane; k < n; k += 32) {
        if (TO_PATCH) arena[d + k] = tr[a + k];
        else tr[a + k] = arena[d + k];
    }
}

// Pack's planes for every chunk of the set in patch order (chunk c holds
// transfers [c per, min((c + 1) per, total)) and its planes start at byte
// 8 c per): byte b of the patch delta at plane b, of the weight at 4 + b.
__global__ void k_shuffle(const int2 *__restrict__ arena, int64_t total, int64_t per, uint8_t *__restrict__ planes) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = g / per, s = c * per, k = g - s, n = min(per, total - s);
        const int2 t = arena[g];
        const uint32_t previous = k ? (uint32_t)arena[g - 1].x : 0u;
        const uint32_t delta = (uint32_t)t.x - previous, weight = (uint32_t)t.y;
        uint8_t *base = planes + kTransferBytes * s + k;
#pragma unroll
        for (int b = 0; b < 4; b++) {
            base[b * n] = (uint8_t)(delta >> (8 * b));
            base[(4 + b) * n] = (uint8_t)(weight >> (8 * b));
        }
    }
}

// The chunk that holds transfer g: the last k < nchunks with starts[k] <= g
// (an empty chunk shares its start with the next).
__device__ __forceinline__ int64_t chunk_of(const int64_t *__restrict__ starts, int64_t nchunks, int64_t g) {
    int64_t lo = 0, hi = nchunks - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (starts[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Every transfer's patch delta out of its chunk's planes.
__global__ void k_plane_deltas(const uint8_t *__restrict__ planes, const int64_t *__restrict__ starts, int64_t nchunks,
                               int64_t total, uint32_t *__restrict__ delta) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = chunk_of(starts, nchunks, g), s = starts[c], n = starts[c + 1] - s;
        const uint8_t *base = planes + kTransferBytes * s + (g - s);
        delta[g] = (uint32_t)base[0] | (uint32_t)base[n] << 8 | (uint32_t)base[2 * n] << 16 |
                   (uint32_t)base[3 * n] << 24;
    }
}

// After the inclusive scan of the deltas (sum[g], wrapping): a transfer's
// patch is its sum less the sum before its chunk, its weight comes from
// planes 4..7.  A patch outside [0, patch_count) sets *bad.
__global__ void k_plane_finish(const uint8_t *__restrict__ planes, const int64_t *__restrict__ starts,
                               int64_t nchunks, int64_t total, const uint32_t *__restrict__ sum, int32_t patch_count,
                               int2 *__restrict__ arena, uint32_t *__restrict__ bad) {
    bool out_of_range = false;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = chunk_of(starts, nchunks, g), s = starts[c], n = starts[c + 1] - s;
        const uint32_t patch = sum[g] - (s > 0 ? sum[s - 1] : 0u);
        const uint8_t *base = planes + kTransferBytes * s + 4 * n + (g - s);
        const uint32_t weight = (uint32_t)base[0] | (uint32_t)base[n] << 8 | (uint32_t)base[2 * n] << 16 |
                                (uint32_t)base[3 * n] << 24;
        out_of_range |= patch >= (uint32_t)patch_count;
        arena[g] = make_int2((int32_t)patch, (int32_t)weight);
    }
    if (__any_sync(0xffffffffu, out_of_range) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
}

}  // namespace

// ---- Host orchestration -------------------------------------------------------

namespace {

// Device memory of one codec call, released at scope exit (the call has
// waited for its stream by then).
struct Scratch {
    std::vector<void *> blocks;
    template <class T>
    cudaError_t get(T **p, size_t bytes) {
        void *q = nullptr;
        const cudaError_t e = cudaMalloc(&q, bytes ? bytes : 1);
        if (e == cudaSuccess) blocks.push_back(q);
        *p = static_cast<T *>(q);
        return e;
    }
    void release(void *q) {
        for (void *&b : blocks)
            if (b == q) {
                cudaFree(b);
                b = nullptr;
            }
    }
    ~Scratch() {
        for (void *q : blocks)
            if (q) cudaFree(q);
    }
};

int device_sms(int device) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return sms > 0 ? sms : 148;
}

// A set decoded onto the device: patch p's list is arena[offsets[p] ..
// offsets[p + 1]).
struct DecodedSet {
    std::vector<int32_t> counts;
    std::vector<int64_t> offsets;
    int32_t max = 0;
    int64_t total = 0;
    int2 *arena = nullptr;  // in the caller's Scratch
};

// ReadPacked (TransferSetCodec.cs:215-297) onto ctx's device.  VRAD_OK,
// VRAD_ERR_FORMAT (the reference's null; *why says which check), or
// VRAD_ERR_CUDA with *err set.
int32_t decode_packed(vrad_ctx *ctx, const uint8_t *index, int64_t index_len, const uint8_t *packed,
                      const int64_t *sizes, int64_t nchunks, int32_t patch_count, Scratch &mem, DecodedSet &out,
                      cudaError_t &err, const char *&why) {
    err = cudaSuccess;
    if (!read_index(index, index_len, patch_count, out.counts, out.max, out.total)) {
        why = "the index does not fit the patch count, or its counts do not add up";
        return VRAD_ERR_FORMAT;
    }
    out.offsets.assign((size_t)patch_count + 1, 0);
    for (int32_t p = 0; p < patch_count; p++) out.offsets[(size_t)p + 1] = out.offsets[(size_t)p] + out.counts[(size_t)p];
    // Every chunk's count from its first four bytes: its place in the set.
    std::vector<int64_t> at((size_t)nchunks + 1, 0), starts((size_t)nchunks + 1, 0);
    for (int64_t k = 0; k < nchunks; k++) {
        if (sizes[k] < 4) {
            why = "a packed chunk shorter than its count";
            return VRAD_ERR_FORMAT;
        }
        const int64_t n = (int32_t)get_u32(packed + at[(size_t)k]);
        if (n < 0 || n > kArrayMaxLength / kTransferBytes) {
            why = "a packed chunk's count out of range";
            return VRAD_ERR_FORMAT;
        }
        at[(size_t)k + 1] = at[(size_t)k] + sizes[k];
        starts[(size_t)k + 1] = starts[(size_t)k] + n;
    }
    if (starts[(size_t)nchunks] != out.total) {
        why = "the chunks' counts do not add up to the index's total";
        return VRAD_ERR_FORMAT;
    }
    if (out.total == 0) return VRAD_OK;
    // Inflate on the host's threads, a chunk to a thread, each into its
    // planes' place in one staging buffer.
    const int64_t T = out.total;
    uvector<uint8_t> planes((size_t)(kTransferBytes * T));
    std::atomic<int> failed{0};
    parallel_for(nchunks, 1, [&](int64_t k) {
        const int64_t n = starts[(size_t)k + 1] - starts[(size_t)k];
        if (!inflate_exact(packed + at[(size_t)k] + 4, sizes[k] - 4, planes.data() + kTransferBytes * starts[(size_t)k],
                           kTransferBytes * n))
            failed.store(1, std::memory_order_relaxed);
    });
    if (failed.load()) {
        why = "a packed chunk does not inflate to exactly its count";
        return VRAD_ERR_FORMAT;
    }
    // The device: deltas out of the planes, their wrapping prefix sum, then
    // each transfer's patch and weight, checked against the patch count.
    cudaStream_t s = ctx->stream;
    uint8_t *d_planes = nullptr;
    int64_t *d_starts = nullptr;
    uint32_t *d_sum = nullptr, *d_bad = nullptr;
    void *d_tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaError_t e = mem.get(&d_planes, (size_t)(kTransferBytes * T));
    if (e == cudaSuccess) e = mem.get(&d_starts, sizeof(int64_t) * ((size_t)nchunks + 1));
    if (e == cudaSuccess) e = mem.get(&d_sum, sizeof(uint32_t) * (size_t)T);
    if (e == cudaSuccess) e = mem.get(&out.arena, sizeof(int2) * (size_t)T);
    if (e == cudaSuccess) e = mem.get(&d_bad, sizeof(uint32_t));
    if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, d_sum, d_sum, (int)T, s);
    if (e == cudaSuccess) e = mem.get(&d_tmp, tmp_bytes);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_planes, planes.data(), (size_t)(kTransferBytes * T), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_starts, starts.data(), sizeof(int64_t) * ((size_t)nchunks + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, sizeof(uint32_t), s);
    const int sms = device_sms(ctx->device);
    if (e == cudaSuccess) {
        k_plane_deltas<<<codec_grid(T, sms), kCodecBlock, 0, s>>>(d_planes, d_starts, nchunks, T, d_sum);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(d_tmp, tmp_bytes, d_sum, d_sum, (int)T, s);
    if (e == cudaSuccess) {
        k_plane_finish<<<codec_grid(T, sms), kCodecBlock, 0, s>>>(d_planes, d_starts, nchunks, T, d_sum, patch_count,
                                                                   out.arena, d_bad);
        e = cudaGetLastError();
    }
    uint32_t bad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = wait_stream(s);
    if (e != cudaSuccess) {
        err = e;
        why = "transfer decode";
        return VRAD_ERR_CUDA;
    }
    mem.release(d_planes);
    mem.release(d_sum);
    mem.release(d_tmp);
    if (bad) {
        why = "a transfer names a patch out of range";
        return VRAD_ERR_FORMAT;
    }
    return VRAD_OK;
}

// The bounce's transfer lists in patch order on the device (arena, in
// mem), with their host offsets and counts.
cudaError_t lists_by_patch(vrad_ctx *ctx, Scratch &mem, DecodedSet &set) {
    BounceBuffers &b = ctx->bounce;
    const int32_t R = b.nreceivers, P = b.npatches;
    cudaStream_t s = ctx->stream;
    std::vector<int64_t> off((size_t)R + 1, 0);
    cudaError_t e = cudaSuccess;
    if (R) e = cudaMemcpyAsync(off.data(), b.tr_off, sizeof(int64_t) * ((size_t)R + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = wait_stream(s);
    if (e != cudaSuccess) return e;
    set.counts.assign((size_t)P, 0);
    for (int32_t r = 0; r < R; r++) set.counts[(size_t)b.h_recv[(size_t)r]] = (int32_t)(off[(size_t)r + 1] - off[(size_t)r]);
    set.offsets.assign((size_t)P + 1, 0);
    set.max = 0;
    for (int32_t p = 0; p < P; p++) {
        set.offsets[(size_t)p + 1] = set.offsets[(size_t)p] + set.counts[(size_t)p];
        set.max = std::max(set.max, set.counts[(size_t)p]);
    }
    set.total = set.offsets[(size_t)P];
    if (set.total == 0) return cudaSuccess;
    int64_t *d_poff = nullptr;
    e = mem.get(&set.arena, sizeof(int2) * (size_t)set.total);
    if (e == cudaSuccess) e = mem.get(&d_poff, sizeof(int64_t) * ((size_t)P + 1));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_poff, set.offsets.data(), sizeof(int64_t) * ((size_t)P + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        k_reorder_lists<true><<<(unsigned)(((int64_t)R * 32 + kCodecBlock - 1) / kCodecBlock), kCodecBlock, 0, s>>>(
            R, b.recv, b.tr_off, d_poff, b.tr, set.arena);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = wait_stream(s);
    return e;
}

}  // namespace

}  // namespace vrad

// ---- The C ABI ------------------------------------------------------------------

using namespace vrad;

extern "C" int32_t vrad_transfer_index(const int64_t *offsets, int32_t npatches, uint8_t *out, int64_t capacity) {
    if (!offsets || !out || npatches < 0) return vrad_fail(nullptr, VRAD_ERR_ARG, "null argument");
    const int64_t need = 20 + 4 * (int64_t)npatches;
    if (capacity < need) return vrad_fail(nullptr, VRAD_ERR_ARG, "the index takes %lld bytes", (long long)need);
    int32_t max = 0;
    for (int32_t p = 0; p < npatches; p++) {
        const int64_t c = offsets[p + 1] - offsets[p];
        if (c < 0 || c > INT32_MAX) return vrad_fail(nullptr, VRAD_ERR_ARG, "patch %d's list has %lld transfers", p, (long long)c);
        max = std::max(max, (int32_t)c);
        put_u32(out + 20 + 4 * (int64_t)p, (uint32_t)c);
    }
    put_u32(out, VRAD_TRANSFER_MAGIC);
    put_u32(out + 4, (uint32_t)npatches);
    put_u32(out + 8, (uint32_t)max);
    put_i64(out + 12, offsets[npatches] - offsets[0]);
    return VRAD_OK;
}

extern "C" int64_t vrad_transfer_pack_bound(int64_t len) { return len < 0 ? 0 : 4 + deflate_room(len); }

extern "C" int32_t vrad_transfer_pack(const uint8_t *chunk, int64_t len, uint8_t *out, int64_t capacity,
                                      int64_t *written) {
    if ((!chunk && len) || !out || !written || len < 0 || len % kTransferBytes)
        return vrad_fail(nullptr, VRAD_ERR_ARG, "a chunk is whole transfers of 8 bytes");
    const int64_t n = len / kTransferBytes;
    if (n > INT32_MAX) return vrad_fail(nullptr, VRAD_ERR_ARG, "a chunk holds at most 2^31 - 1 transfers");
    if (capacity < 4) return vrad_fail(nullptr, VRAD_ERR_ARG, "no room for the count");
    std::vector<uint8_t> planes((size_t)len);
    shuffle_host(chunk, n, planes.data());
    put_u32(out, (uint32_t)n);
    const int64_t z = deflate_fast(planes.data(), len, out + 4, capacity - 4);
    if (z < 0) return vrad_fail(nullptr, VRAD_ERR_ARG, "%lld bytes are not room enough", (long long)capacity);
    *written = 4 + z;
    return VRAD_OK;
}

extern "C" int32_t vrad_transfer_unpack(const uint8_t *packed, int64_t len, uint8_t *out, int64_t capacity,
                                        int64_t *written) {
    if ((!packed && len) || !written || len < 0) return vrad_fail(nullptr, VRAD_ERR_ARG, "null argument");
    if (len < 4) return vrad_fail(nullptr, VRAD_ERR_FORMAT, "shorter than a packed chunk's count");
    const int64_t n = (int32_t)get_u32(packed);
    if (n < 0 || n > kArrayMaxLength / kTransferBytes)
        return vrad_fail(nullptr, VRAD_ERR_FORMAT, "a packed chunk's count out of range");
    if (capacity < kTransferBytes * n || (!out && n))
        return vrad_fail(nullptr, VRAD_ERR_ARG, "the chunk takes %lld bytes", (long long)(kTransferBytes * n));
    // Uninitialised: junk that claims a large count fails in the inflate
    // without touching the pages.
    uvector<uint8_t> planes((size_t)(kTransferBytes * n));
    if (!inflate_exact(packed + 4, len - 4, planes.data(), kTransferBytes * n))
        return vrad_fail(nullptr, VRAD_ERR_FORMAT, "the stream does not inflate to exactly its count");
    unshuffle_host(planes.data(), n, out);
    *written = kTransferBytes * n;
    return VRAD_OK;
}

namespace {

// The transfer count of the context's current set, and whether it has one.
int32_t current_total(vrad_ctx *ctx, int64_t &total) {
    BounceBuffers &b = ctx->bounce;
    if (!b.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "no bounce uploaded");
    if (!b.lists_ready) return vrad_fail(ctx, VRAD_ERR_ARG, "no transfers yet: bounce a light pass or install a set");
    total = b.ntransfers;
    return VRAD_OK;
}

}  // namespace

extern "C" int32_t vrad_transfer_export_size(vrad_ctx *ctx, int64_t max_chunk_bytes, int64_t *index_len,
                                             int64_t *nchunks, int64_t *packed_bound) {
    if (!ctx || !index_len || !nchunks || !packed_bound) return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    int64_t T = 0;
    const int32_t rc = current_total(ctx, T);
    if (rc != VRAD_OK) return rc;
    const int64_t per = per_chunk(max_chunk_bytes);
    const int64_t K = (T + per - 1) / per;
    *index_len = 20 + 4 * (int64_t)ctx->bounce.npatches;
    *nchunks = K;
    *packed_bound = K == 0 ? 0 : (K - 1) * (4 + deflate_room(kTransferBytes * per)) +
                                     4 + deflate_room(kTransferBytes * (T - (K - 1) * per));
    return VRAD_OK;
}

extern "C" int32_t vrad_transfer_export(vrad_ctx *ctx, int64_t max_chunk_bytes, uint8_t *index,
                                        int64_t index_capacity, uint8_t *packed, int64_t packed_capacity,
                                        int64_t *chunk_sizes, int64_t chunk_capacity, int64_t *packed_len) {
    if (!ctx || !index || !packed_len || (chunk_capacity > 0 && !chunk_sizes))
        return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    int64_t T0 = 0;
    int32_t rc = current_total(ctx, T0);
    if (rc != VRAD_OK) return rc;
    cudaError_t e = cudaSetDevice(ctx->device);
    settle_direct(ctx);
    if (e == cudaSuccess) e = quiesce(ctx);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "waiting for the context's kernels");
    const int32_t P = ctx->bounce.npatches;
    if (index_capacity < 20 + 4 * (int64_t)P) return vrad_fail(ctx, VRAD_ERR_ARG, "no room for the index");
    Scratch mem;
    DecodedSet set;
    e = lists_by_patch(ctx, mem, set);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "transfer lists in patch order");
    rc = vrad_transfer_index(set.offsets.data(), P, index, index_capacity);
    if (rc != VRAD_OK) return vrad_fail(ctx, rc, "transfer index");
    const int64_t T = set.total, per = per_chunk(max_chunk_bytes);
    const int64_t K = (T + per - 1) / per;
    if (chunk_capacity < K) return vrad_fail(ctx, VRAD_ERR_ARG, "%lld chunks, room for %lld", (long long)K, (long long)chunk_capacity);
    *packed_len = 0;
    if (T == 0) return VRAD_OK;
    // The planes on the device, then to the host.
    uint8_t *d_planes = nullptr;
    e = mem.get(&d_planes, (size_t)(kTransferBytes * T));
    if (e == cudaSuccess) {
        k_shuffle<<<codec_grid(T, device_sms(ctx->device)), kCodecBlock, 0, ctx->stream>>>(set.arena, T, per, d_planes);
        e = cudaGetLastError();
    }
    uvector<uint8_t> planes((size_t)(kTransferBytes * T));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(planes.data(), d_planes, (size_t)(kTransferBytes * T), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = wait_stream(ctx->stream);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "transfer planes");
    // Each chunk deflated by a host thread into its own block, then the
    // blocks copied back to back.
    std::vector<std::vector<uint8_t>> blocks((size_t)K);
    std::atomic<int> failed{0};
    parallel_for(K, 1, [&](int64_t k) {
        const int64_t s = k * per, n = std::min(per, T - s);
        std::vector<uint8_t> &out = blocks[(size_t)k];
        out.resize((size_t)(4 + deflate_room(kTransferBytes * n)));
        put_u32(out.data(), (uint32_t)n);
        const int64_t z = deflate_fast(planes.data() + kTransferBytes * s, kTransferBytes * n, out.data() + 4,
                                       (int64_t)out.size() - 4);
        if (z < 0) failed.store(1, std::memory_order_relaxed);
        else out.resize((size_t)(4 + z));
    });
    if (failed.load()) return vrad_fail(ctx, VRAD_ERR_ARG, "deflate failed");
    std::vector<int64_t> at((size_t)K + 1, 0);
    for (int64_t k = 0; k < K; k++) at[(size_t)k + 1] = at[(size_t)k] + (int64_t)blocks[(size_t)k].size();
    *packed_len = at[(size_t)K];
    if (!packed || packed_capacity < at[(size_t)K])
        return vrad_fail(ctx, VRAD_ERR_ARG, "the packed chunks take %lld bytes", (long long)at[(size_t)K]);
    parallel_for(K, 1, [&](int64_t k) {
        std::memcpy(packed + at[(size_t)k], blocks[(size_t)k].data(), blocks[(size_t)k].size());
        chunk_sizes[k] = (int64_t)blocks[(size_t)k].size();
    });
    return VRAD_OK;
}

namespace {

bool packed_args(const uint8_t *index, const uint8_t *packed, const int64_t *sizes, int64_t nchunks) {
    return index && nchunks >= 0 && (nchunks == 0 || (packed && sizes));
}

int32_t decode_failed(vrad_ctx *ctx, int32_t rc, cudaError_t err, const char *why) {
    return rc == VRAD_ERR_CUDA ? vrad_cuda_fail(ctx, err, why) : vrad_fail(ctx, rc, "%s", why);
}

}  // namespace

extern "C" int32_t vrad_transfer_read_packed(vrad_ctx *ctx, const uint8_t *index, int64_t index_len,
                                             const uint8_t *packed, const int64_t *chunk_sizes, int64_t nchunks,
                                             int32_t patch_count, int64_t *offsets, vrad_transfer *transfers,
                                             int64_t capacity, int64_t *total) {
    if (!ctx || !offsets || !total || patch_count < 0 || !packed_args(index, packed, chunk_sizes, nchunks))
        return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "cudaSetDevice");
    Scratch mem;
    DecodedSet set;
    const char *why = "";
    const int32_t rc = decode_packed(ctx, index, index_len, packed, chunk_sizes, nchunks, patch_count, mem, set, e, why);
    if (rc != VRAD_OK) return decode_failed(ctx, rc, e, why);
    std::memcpy(offsets, set.offsets.data(), sizeof(int64_t) * ((size_t)patch_count + 1));
    *total = set.total;
    if (!transfers || set.total == 0) return VRAD_OK;
    if (capacity < set.total)
        return vrad_fail(ctx, VRAD_ERR_ARG, "%lld transfers, room for %lld", (long long)set.total, (long long)capacity);
    static_assert(sizeof(vrad_transfer) == sizeof(int2), "a transfer is (patch, weight bits)");
    e = cudaMemcpyAsync(transfers, set.arena, sizeof(int2) * (size_t)set.total, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = wait_stream(ctx->stream);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "transfer download");
    return VRAD_OK;
}

extern "C" int32_t vrad_transfer_install(vrad_ctx *ctx, const uint8_t *index, int64_t index_len,
                                         const uint8_t *packed, const int64_t *chunk_sizes, int64_t nchunks) {
    if (!ctx || !packed_args(index, packed, chunk_sizes, nchunks)) return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    BounceBuffers &b = ctx->bounce;
    if (!b.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "no bounce uploaded");
    cudaError_t e = cudaSetDevice(ctx->device);
    settle_direct(ctx);
    if (e == cudaSuccess) e = quiesce(ctx);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "waiting for the context's kernels");
    Scratch mem;
    DecodedSet set;
    const char *why = "";
    const int32_t rc = decode_packed(ctx, index, index_len, packed, chunk_sizes, nchunks, b.npatches, mem, set, e, why);
    if (rc != VRAD_OK) return decode_failed(ctx, rc, e, why);
    // The set must be one this bounce could have built: lists on receivers
    // only, no more transfers than candidate pairs.
    const int32_t R = b.nreceivers, P = b.npatches;
    std::vector<char> receives((size_t)P, 0);
    for (int32_t r = 0; r < R; r++) receives[(size_t)b.h_recv[(size_t)r]] = 1;
    for (int32_t p = 0; p < P; p++)
        if (set.counts[(size_t)p] > 0 && !receives[(size_t)p])
            return vrad_fail(ctx, VRAD_ERR_FORMAT, "patch %d has transfers but receives none in this bounce", p);
    if (set.total > b.ncand)
        return vrad_fail(ctx, VRAD_ERR_FORMAT, "%lld transfers, more than the %lld candidate pairs", (long long)set.total,
                         (long long)b.ncand);
    if (set.max > kMaxTransfersPerReceiver)
        return vrad_fail(ctx, VRAD_ERR_FORMAT, "a list of %d transfers, longer than any build makes", set.max);
    // Receiver order: the offsets on the host, the lists moved on the device,
    // then the gather's slices.
    std::vector<int64_t> off((size_t)R + 1, 0);
    for (int32_t r = 0; r < R; r++) off[(size_t)r + 1] = off[(size_t)r] + set.counts[(size_t)b.h_recv[(size_t)r]];
    cudaStream_t s = ctx->stream;
    int64_t *d_poff = nullptr;
    e = mem.get(&d_poff, sizeof(int64_t) * ((size_t)P + 1));
    if (e == cudaSuccess && R)
        e = cudaMemcpyAsync(b.tr_off, off.data(), sizeof(int64_t) * ((size_t)R + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_poff, set.offsets.data(), sizeof(int64_t) * ((size_t)P + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && R && set.total) {
        k_reorder_lists<false><<<(unsigned)(((int64_t)R * 32 + kCodecBlock - 1) / kCodecBlock), kCodecBlock, 0, s>>>(
            R, b.recv, b.tr_off, d_poff, b.tr, set.arena);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = launch_sell(b, s);
    if (e == cudaSuccess) e = wait_stream(s);
    if (e != cudaSuccess) {
        b.lists_ready = false;
        b.installed = false;
        return vrad_cuda_fail(ctx, e, "transfer install");
    }
    b.ntransfers = set.total;
    b.installed = true;
    b.lists_ready = true;
    return VRAD_OK;
}
