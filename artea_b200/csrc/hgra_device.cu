// HGRA v1 snapshot restored straight to the device.
//
// The snapshot (index/persistence/hierarchical_graph_file_manager.hpp:15-39)
// is a header and one variable-length record per vertex: highest level, then
// for each level from it down to 0 a count and that many neighbour ids.
// Restore (hierarchical_graph_file_manager.hpp:152-300) buckets vertices by
// highest level in vid order and lays each group's rows out as one CSR.
//
// Here the records stream in fixed chunks through two pinned buffers into a
// raw copy in device memory. While a chunk is in flight the host walks its
// record headers only (highest levels and counts; the ids are skipped), which
// gives the vertex table, the CSR offsets and, for every CSR row, where its
// ids sit in the raw copy. One kernel then moves every row's ids into place
// and checks them, so the ids cross the host once (the file read) and are
// never parsed there. Layout, accepted files and status codes are those of
// artea_gpu_hgra_read followed by artea_gpu_index_create.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

using namespace artea_gpu;

namespace {

constexpr uint32_t kMagic = 0x48475241u;
constexpr uint32_t kVersion = 1u;
constexpr uint32_t kNone = 0xffffffffu;
constexpr size_t kChunkWords = size_t(1) << 23;   // 32 MiB per pinned buffer

constexpr uint32_t kFlagBadId = 1u;      // an id >= num_vertices (the reader's EIO)
constexpr uint32_t kFlagOffLevel = 2u;   // an id whose vertex is not on the row's level (validation's EGRAPH)

// One warp per CSR row (grid-stride): copies the row's ids from the raw
// records to their CSR position and flags ids out of range or off the row's
// level. src/dst/len come from the host's header walk, which checked that
// every row lies inside the raw copy and inside the CSR array.
__global__ void hgra_rows_kernel(const uint32_t* __restrict__ raw, const unsigned long long* __restrict__ src,
                                 const unsigned long long* __restrict__ dst,
                                 const unsigned long long* __restrict__ len_lvl, unsigned long long rows,
                                 const uint2* __restrict__ vinfo, uint32_t n, uint32_t* __restrict__ nbrs,
                                 uint32_t* flags) {
    const int lane = threadIdx.x & 31;
    const unsigned long long wpb = blockDim.x >> 5;
    const unsigned long long warps = static_cast<unsigned long long>(gridDim.x) * wpb;
    uint32_t bad = 0;
    for (unsigned long long r = blockIdx.x * wpb + (threadIdx.x >> 5); r < rows; r += warps) {
        const unsigned long long m = len_lvl[r];
        const uint32_t len = static_cast<uint32_t>(m);
        const uint32_t lvl = static_cast<uint32_t>(m >> 32);
        const unsigned long long s = src[r], d = dst[r];
        for (uint32_t i = lane; i < len; i += 32) {
            const uint32_t id = raw[s + i];
            nbrs[d + i] = id;
            if (id >= n) {
                bad |= kFlagBadId;
            } else {
                const uint32_t h = vinfo[id].x;
                if (h == kNone || h < lvl) bad |= kFlagOffLevel;
            }
        }
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (lane == 0 && bad) atomicOr(flags, bad);
}

// Host resources of one restore; released on every exit path.
struct Restore {
    FILE* fp = nullptr;
    cudaStream_t stream = nullptr;
    uint32_t* pinned[2] = {nullptr, nullptr};
    cudaEvent_t copied[2] = {nullptr, nullptr};
    uint32_t* d_raw = nullptr;
    unsigned long long* d_src = nullptr;
    unsigned long long* d_dst = nullptr;
    unsigned long long* d_len = nullptr;
    uint32_t* d_flags = nullptr;
    int device = -1;   // set once device resources exist
    ~Restore() {
        if (device < 0) {
            if (fp) std::fclose(fp);
            return;
        }
        DeviceGuard guard(device);
        if (stream) cudaStreamSynchronize(stream);
        if (fp) std::fclose(fp);
        for (int i = 0; i < 2; ++i) {
            if (pinned[i]) cudaFreeHost(pinned[i]);
            if (copied[i]) cudaEventDestroy(copied[i]);
        }
        dev_free(d_raw);
        dev_free(d_src);
        dev_free(d_dst);
        dev_free(d_len);
        dev_free(d_flags);
        if (stream) cudaStreamDestroy(stream);
    }
};

}  // namespace

// CUDA_TRY for code that holds a partly built index: releases it first.
#define CUDA_TRY_IX(expr)                                                                          \
    do {                                                                                           \
        cudaError_t _e = (expr);                                                                   \
        if (_e != cudaSuccess)                                                                     \
            return cleanup(fail(ARTEA_GPU_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(_e))); \
    } while (0)

extern "C" int artea_gpu_index_create_from_hgra(const char* path, const float* vectors, uint32_t num_vectors,
                                                uint32_t dim, int device, artea_gpu_index** out) {
    if (!path || !out) return fail(ARTEA_GPU_EINVAL, "null argument");
    *out = nullptr;
    Restore rs;
    rs.fp = std::fopen(path, "rb");
    if (!rs.fp) return fail(ARTEA_GPU_EIO, std::string("cannot open ") + path);
    std::fseek(rs.fp, 0, SEEK_END);
    const long bytes = std::ftell(rs.fp);
    std::fseek(rs.fp, 0, SEEK_SET);
    if (bytes < 28 || bytes % 4 != 0)
        return fail(ARTEA_GPU_EIO, std::string("truncated or misaligned snapshot ") + path);
    uint32_t hdr[7];
    if (std::fread(hdr, 4, 7, rs.fp) != 7) return fail(ARTEA_GPU_EIO, std::string("short read of ") + path);
    if (hdr[0] != kMagic) return fail(ARTEA_GPU_EIO, "bad HGRA magic");
    if (hdr[1] != kVersion) return fail(ARTEA_GPU_EIO, "unsupported HGRA version");
    const uint32_t n = hdr[2], top = hdr[3], ul = hdr[4], bl = hdr[5], entry = hdr[6];
    if (top == kNone || (entry != kNone && entry >= n && n != 0)) return fail(ARTEA_GPU_EIO, "invalid HGRA header");
    if (top >= 64) return fail(ARTEA_GPU_EIO, "HGRA top level above 63 is not supported");
    const uint64_t rec_words = static_cast<uint64_t>(bytes) / 4 - 7;
    // Every vertex record holds at least its highest-level word.
    if (rec_words < n) return fail(ARTEA_GPU_EIO, "HGRA truncated at vid " + std::to_string(rec_words));

    artea_gpu_index* ix = nullptr;
    if (n == 0) {
        // hierarchical_graph_file_manager.hpp restores an empty graph.
        if (rec_words != 0) return fail(ARTEA_GPU_EIO, "HGRA has trailing bytes");
        if (int rc = index_begin(0, vectors, num_vectors, dim, device, &ix)) return rc;
        ix->n = 0;
        ix->top = kInvalidLevel;
        ix->entry = entry;
        ix->ul = ul;
        ix->bl = bl;
        *out = ix;
        return ARTEA_GPU_OK;
    }
    if (int rc = index_begin(n, vectors, num_vectors, dim, device, &ix)) return rc;
    auto cleanup = [&](int rc) {
        artea_gpu_index_destroy(ix);
        return rc;
    };
    DeviceGuard guard(device);
    ix->n = n;
    ix->top = top;
    ix->entry = entry;
    ix->ul = ul;
    ix->bl = bl;

    // ---- stream the records to the device, walking their headers ----
    rs.device = device;
    if (int rc = dev_alloc(&rs.d_raw, std::max<uint64_t>(rec_words, 1))) return cleanup(rc);
    if (cudaStreamCreateWithFlags(&rs.stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(ARTEA_GPU_ECUDA, "cannot create stream"));
    for (int i = 0; i < 2; ++i) {
        if (cudaHostAlloc(reinterpret_cast<void**>(&rs.pinned[i]), kChunkWords * 4, cudaHostAllocDefault) !=
                cudaSuccess ||
            cudaEventCreateWithFlags(&rs.copied[i], cudaEventDisableTiming) != cudaSuccess)
            return cleanup(fail(ARTEA_GPU_ENOMEM, "pinned staging buffers unavailable"));
    }
    std::vector<uint32_t> hl(n, kNone);
    std::vector<uint64_t> vrow(n, 0);     // first row of v in file order
    std::vector<uint32_t> rcnt;           // per row in file order: id count
    std::vector<uint64_t> rsrc;           // per row in file order: raw word of its first id
    rcnt.reserve(n);
    rsrc.reserve(n);
    uint64_t gsize[64] = {};
    uint64_t total_ids = 0;
    uint32_t v = 0;        // vertex whose record is being read
    int state = 0;         // 0: highest level next, 1: a count next, 2: skipping a row's ids
    uint32_t lvl = 0;      // level of the next count / the row being skipped
    uint64_t skip = 0;     // ids of the current row still to skip
    std::string err;
    auto row_done = [&]() {
        if (lvl == 0) {
            ++v;
            state = 0;
        } else {
            --lvl;
            state = 1;
        }
    };
    uint64_t chunk = 0;
    for (uint64_t off = 0; off < rec_words && err.empty(); off += kChunkWords, ++chunk) {
        const size_t cw = static_cast<size_t>(std::min<uint64_t>(kChunkWords, rec_words - off));
        const int b = static_cast<int>(chunk & 1);
        if (cudaEventSynchronize(rs.copied[b]) != cudaSuccess)   // the copy that last read this buffer
            return cleanup(fail(ARTEA_GPU_ECUDA, "snapshot upload failed"));
        uint32_t* w = rs.pinned[b];
        if (std::fread(w, 4, cw, rs.fp) != cw) {
            err = std::string("short read of ") + path;
            break;
        }
        CUDA_TRY_IX(cudaMemcpyAsync(rs.d_raw + off, w, cw * 4, cudaMemcpyHostToDevice, rs.stream));
        CUDA_TRY_IX(cudaEventRecord(rs.copied[b], rs.stream));
        size_t i = 0;
        while (i < cw) {
            if (state == 2) {
                const uint64_t k = std::min<uint64_t>(skip, cw - i);
                i += k;
                skip -= k;
                if (skip == 0) row_done();
                continue;
            }
            if (state == 0) {
                if (v >= n) {
                    err = "HGRA has trailing bytes";
                    break;
                }
                const uint32_t h = w[i++];
                hl[v] = h;
                if (h == kNone) {
                    ++v;
                    continue;
                }
                if (h > top) {
                    err = "HGRA vid " + std::to_string(v) + " above top level";
                    break;
                }
                gsize[h]++;
                vrow[v] = rcnt.size();
                lvl = h;
                state = 1;
                continue;
            }
            const uint64_t at = off + i;   // raw word of this count
            const uint32_t cnt = w[i++];
            const uint32_t capacity = lvl == 0 ? bl : ul;
            if (cnt > capacity) {
                err = "HGRA row longer than its level capacity";
                break;
            }
            if (at + 1 + cnt > rec_words) {
                err = "HGRA truncated in a row";
                break;
            }
            rcnt.push_back(cnt);
            rsrc.push_back(at + 1);
            total_ids += cnt;
            if (cnt == 0) {
                row_done();
            } else {
                skip = cnt;
                state = 2;
            }
        }
    }
    if (err.empty() && state == 1) err = "HGRA truncated in vid " + std::to_string(v);
    if (err.empty() && v < n) err = "HGRA truncated at vid " + std::to_string(v);
    CUDA_TRY_IX(cudaStreamSynchronize(rs.stream));
    if (!err.empty()) return cleanup(fail(ARTEA_GPU_EIO, err));

    // ---- vertex table, CSR offsets and the row moves (restore's layout) ----
    const uint32_t groups = top + 1;
    std::vector<uint32_t> vinfo(2ull * n);
    std::vector<uint64_t> gstart(groups + 1, 0);
    for (uint32_t h = 0; h < groups; ++h) gstart[h + 1] = gstart[h] + gsize[h];
    std::vector<uint32_t> order(gstart[groups]);   // vertices bucketed by highest level, vid order
    std::vector<uint64_t> fill(gstart.begin(), gstart.end() - 1);
    for (uint32_t u = 0; u < n; ++u) {
        const uint32_t h = hl[u];
        if (h == kNone) {
            vinfo[2ull * u] = kNone;
            vinfo[2ull * u + 1] = kNone;
            continue;
        }
        vinfo[2ull * u] = h;
        vinfo[2ull * u + 1] = static_cast<uint32_t>(fill[h] - gstart[h]);
        order[fill[h]++] = u;
    }
    uint64_t num_offsets = 0, num_rows = 0;
    for (uint32_t h = 0; h < groups; ++h) {
        num_offsets += gsize[h] * (h + 1ull) + 1;
        num_rows += gsize[h] * (h + 1ull);
    }
    std::vector<uint64_t> offs(num_offsets);
    std::vector<const uint64_t*> gptr(groups);
    std::vector<unsigned long long> jsrc(num_rows), jdst(num_rows), jlen(num_rows);
    {
        uint64_t at = 0, obase = 0, row = 0;
        for (uint32_t h = 0; h < groups; ++h) {
            uint64_t* o = offs.data() + obase;
            gptr[h] = o;
            uint64_t rr = 0;
            for (uint64_t k = gstart[h]; k < gstart[h + 1]; ++k) {
                const uint64_t fr = vrow[order[k]];
                for (uint32_t j = 0; j <= h; ++j, ++row) {
                    const uint32_t cnt = rcnt[fr + j];
                    o[rr++] = at;
                    jsrc[row] = rsrc[fr + j];
                    jdst[row] = at;
                    jlen[row] = cnt | (static_cast<unsigned long long>(h - j) << 32);
                    at += cnt;
                }
            }
            o[rr] = at;
            obase += gsize[h] * (h + 1ull) + 1;
        }
    }
    ix->n_offsets = num_offsets;
    ix->n_nbrs = total_ids;
    if (int rc = dev_alloc(&ix->d_vinfo, n)) return cleanup(rc);
    if (int rc = dev_alloc(&ix->d_offsets, num_offsets)) return cleanup(rc);
    if (int rc = dev_alloc(&ix->d_nbrs, std::max<uint64_t>(total_ids, 1))) return cleanup(rc);
    if (int rc = dev_alloc(&rs.d_flags, 1)) return cleanup(rc);
    CUDA_TRY_IX(cudaMemcpy(ix->d_vinfo, vinfo.data(), sizeof(uint2) * n, cudaMemcpyHostToDevice));
    CUDA_TRY_IX(cudaMemcpy(ix->d_offsets, offs.data(), sizeof(uint64_t) * num_offsets, cudaMemcpyHostToDevice));
    CUDA_TRY_IX(cudaMemset(rs.d_flags, 0, sizeof(uint32_t)));
    {
        uint64_t obase = 0;
        for (uint32_t h = 0; h < groups; ++h) {
            ix->group_ptr[h] = ix->d_offsets + obase;
            obase += gsize[h] * (h + 1ull) + 1;
        }
    }
    if (num_rows) {
        if (int rc = dev_alloc(&rs.d_src, num_rows)) return cleanup(rc);
        if (int rc = dev_alloc(&rs.d_dst, num_rows)) return cleanup(rc);
        if (int rc = dev_alloc(&rs.d_len, num_rows)) return cleanup(rc);
        const size_t jb = sizeof(unsigned long long) * num_rows;
        CUDA_TRY_IX(cudaMemcpy(rs.d_src, jsrc.data(), jb, cudaMemcpyHostToDevice));
        CUDA_TRY_IX(cudaMemcpy(rs.d_dst, jdst.data(), jb, cudaMemcpyHostToDevice));
        CUDA_TRY_IX(cudaMemcpy(rs.d_len, jlen.data(), jb, cudaMemcpyHostToDevice));
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const uint64_t want = (num_rows + 7) / 8;   // 8 warps per block
        const int grid = static_cast<int>(std::min<uint64_t>(want, static_cast<uint64_t>(std::max(sms, 1)) * 16));
        hgra_rows_kernel<<<grid, 256, 0, rs.stream>>>(rs.d_raw, rs.d_src, rs.d_dst, rs.d_len, num_rows, ix->d_vinfo,
                                                      n, ix->d_nbrs, rs.d_flags);
        CUDA_TRY_IX(cudaGetLastError());
    }
    uint32_t flags = 0;
    CUDA_TRY_IX(cudaMemcpyAsync(&flags, rs.d_flags, sizeof(uint32_t), cudaMemcpyDeviceToHost, rs.stream));
    CUDA_TRY_IX(cudaStreamSynchronize(rs.stream));
    dev_free(rs.d_raw);
    // The reader's check first (EIO), then artea_gpu_graph_validate's (EGRAPH).
    if (flags & kFlagBadId) return cleanup(fail(ARTEA_GPU_EIO, "HGRA neighbour id out of range"));
    if (entry >= n) return cleanup(fail(ARTEA_GPU_EGRAPH, "entry point out of range"));
    if (hl[entry] != top) return cleanup(fail(ARTEA_GPU_EGRAPH, "entry point is not on the top level"));
    if (flags & kFlagOffLevel)
        return cleanup(fail(ARTEA_GPU_EGRAPH, "a neighbour id is not on the level of the row that names it"));
    if (int rc = index_finish_l0(ix, vinfo.data(), gptr.data())) return cleanup(rc);
    *out = ix;
    return ARTEA_GPU_OK;
}

extern "C" int artea_gpu_index_download(const artea_gpu_index* ix, uint32_t* vertex_info, uint64_t* offsets,
                                        uint32_t* neighbor_ids) {
    if (!ix || !vertex_info || !offsets || !neighbor_ids) return fail(ARTEA_GPU_EINVAL, "null argument");
    if (ix->n == 0 || ix->top == kInvalidLevel || !ix->d_vinfo) return fail(ARTEA_GPU_EINVAL, "index holds no graph");
    DeviceGuard guard(ix->device);
    CUDA_TRY(cudaMemcpy(vertex_info, ix->d_vinfo, sizeof(uint2) * ix->n, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(offsets, ix->d_offsets, sizeof(uint64_t) * ix->n_offsets, cudaMemcpyDeviceToHost));
    if (ix->n_nbrs)
        CUDA_TRY(cudaMemcpy(neighbor_ids, ix->d_nbrs, sizeof(uint32_t) * ix->n_nbrs, cudaMemcpyDeviceToHost));
    return ARTEA_GPU_OK;
}
