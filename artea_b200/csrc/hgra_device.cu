// HGRA v1 snapshot restored straight to the device.
//
// The snapshot (index/persistence/hierarchical_graph_file_manager.hpp:15-39)
// is a header and one variable-length record per vertex: highest level, then
// for each level from it down to 0 a count and that many neighbour ids.
// Restore (hierarchical_graph_file_manager.hpp:152-300) buckets vertices by
// highest level in vid order and lays each group's rows out as one CSR.
//
// Here reader threads pread the records in fixed chunks into pinned buffers,
// and each chunk is copied into a raw copy of the records in device memory.
// While a chunk's copy is in flight the calling thread walks its record
// headers only (highest levels and counts; the ids are skipped), which gives
// the vertex table, the CSR offsets and, for every CSR row, where its ids sit
// in the raw copy. One kernel then moves every row's ids into place and
// checks them, so the ids cross the host once (the file read) and are never
// parsed there. Layout, accepted files and status codes are those of
// artea_gpu_hgra_read followed by artea_gpu_index_create.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

using namespace artea_gpu;

namespace {

constexpr uint32_t kMagic = 0x48475241u;
constexpr uint32_t kVersion = 1u;
constexpr uint32_t kNone = 0xffffffffu;
constexpr size_t kChunkWords = size_t(1) << 22;   // 16 MiB per pinned buffer
constexpr int kReaders = 4;                         // reader threads, one pinned buffer each
constexpr uint64_t kFree = ~0ull;

constexpr uint32_t kFlagBadId = 1u;      // an id >= num_vertices (the reader's EIO)
constexpr uint32_t kFlagOffLevel = 2u;   // an id whose vertex is not on the row's level (validation's EGRAPH)

constexpr uint32_t kGroupsMax = 64;

// The CSR's row groups: group h holds the flattened rows [row_begin[h],
// row_begin[h + 1]) and its offsets start at offsets + obase[h].
struct RowGroups {
    unsigned long long row_begin[kGroupsMax + 1];
    unsigned long long obase[kGroupsMax];
    uint32_t groups;
};

// One warp per CSR row (grid-stride): copies the row's ids from the raw
// records to their CSR position and flags ids out of range or off the row's
// level. A row's destination and length come from the CSR offsets, its level
// from its position in the group, its source from src (the host's header walk
// checked that every row lies inside the raw copy).
__global__ void hgra_rows_kernel(const uint32_t* __restrict__ raw, const unsigned long long* __restrict__ src,
                                 RowGroups gr, const uint64_t* __restrict__ offsets,
                                 const uint2* __restrict__ vinfo, uint32_t n, uint32_t* __restrict__ nbrs,
                                 uint32_t* flags) {
    const int lane = threadIdx.x & 31;
    const unsigned long long wpb = blockDim.x >> 5;
    const unsigned long long warps = static_cast<unsigned long long>(gridDim.x) * wpb;
    const unsigned long long rows = gr.row_begin[gr.groups];
    uint32_t bad = 0;
    uint32_t h = 0;   // the warp's rows only grow, so its group index only moves forward
    for (unsigned long long r = blockIdx.x * wpb + (threadIdx.x >> 5); r < rows; r += warps) {
        while (r >= gr.row_begin[h + 1]) ++h;
        const unsigned long long rr = r - gr.row_begin[h];
        const uint64_t* o = offsets + gr.obase[h];
        const unsigned long long d = o[rr];
        const uint32_t len = static_cast<uint32_t>(o[rr + 1] - d);
        const uint32_t lvl = h - static_cast<uint32_t>(rr % (h + 1ull));
        const unsigned long long s = src[r];
        for (uint32_t i = lane; i < len; i += 32) {
            const uint32_t id = raw[s + i];
            nbrs[d + i] = id;
            if (id >= n) {
                bad |= kFlagBadId;
            } else {
                const uint32_t vh = vinfo[id].x;
                if (vh == kNone || vh < lvl) bad |= kFlagOffLevel;
            }
        }
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (lane == 0 && bad) atomicOr(flags, bad);
}

// Host resources of one restore; released on every exit path.
struct Restore {
    int fd = -1;
    cudaStream_t stream = nullptr;
    uint32_t* pinned[kReaders] = {};
    cudaEvent_t copied[kReaders] = {};
    uint32_t* d_raw = nullptr;
    unsigned long long* d_src = nullptr;
    uint32_t* d_flags = nullptr;
    int device = -1;   // set once device resources exist
    // Reader t fills buffer t with chunks t, t + kReaders, ... in order, each
    // once the walk has released the buffer (holds[t] == kFree).
    std::vector<std::thread> readers;
    std::mutex mu;
    std::condition_variable cv;
    uint64_t holds[kReaders];
    bool read_ok[kReaders] = {};
    bool stop = false;

    Restore() {
        for (auto& h : holds) h = kFree;
    }

    void stop_readers() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        for (auto& t : readers)
            if (t.joinable()) t.join();
        readers.clear();
    }
    ~Restore() {
        stop_readers();
        if (device >= 0) {
            DeviceGuard guard(device);
            if (stream) cudaStreamSynchronize(stream);
            for (int i = 0; i < kReaders; ++i) {
                if (pinned[i]) cudaFreeHost(pinned[i]);
                if (copied[i]) cudaEventDestroy(copied[i]);
            }
            dev_free(d_raw);
            dev_free(d_src);
            dev_free(d_flags);
            if (stream) cudaStreamDestroy(stream);
        }
        if (fd >= 0) close(fd);
    }
};

bool pread_all(int fd, void* dst, size_t bytes, off_t at) {
    char* p = static_cast<char*>(dst);
    while (bytes) {
        const ssize_t k = pread(fd, p, bytes, at);
        if (k < 0 && errno == EINTR) continue;
        if (k <= 0) return false;
        p += k;
        bytes -= static_cast<size_t>(k);
        at += k;
    }
    return true;
}

// Reader thread t: chunks t, t + kReaders, ... of the records (which start
// after the 28-byte header) into pinned buffer t.
void read_chunks(Restore* rs, int t, uint64_t nchunks, uint64_t rec_words) {
    for (uint64_t c = static_cast<uint64_t>(t); c < nchunks; c += kReaders) {
        {
            std::unique_lock<std::mutex> lk(rs->mu);
            rs->cv.wait(lk, [&] { return rs->stop || rs->holds[t] == kFree; });
            if (rs->stop) return;
        }
        const uint64_t off = c * kChunkWords;
        const size_t bytes = static_cast<size_t>(std::min<uint64_t>(kChunkWords, rec_words - off)) * 4;
        const bool ok = pread_all(rs->fd, rs->pinned[t], bytes, static_cast<off_t>(28 + off * 4));
        {
            std::lock_guard<std::mutex> lk(rs->mu);
            rs->holds[t] = c;
            rs->read_ok[t] = ok;
        }
        rs->cv.notify_all();
    }
}

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
    rs.fd = open(path, O_RDONLY | O_CLOEXEC);
    if (rs.fd < 0) return fail(ARTEA_GPU_EIO, std::string("cannot open ") + path);
    struct stat st;
    if (fstat(rs.fd, &st) != 0) return fail(ARTEA_GPU_EIO, std::string("cannot stat ") + path);
    const uint64_t bytes = static_cast<uint64_t>(st.st_size);
    if (bytes < 28 || bytes % 4 != 0)
        return fail(ARTEA_GPU_EIO, std::string("truncated or misaligned snapshot ") + path);
    uint32_t hdr[7];
    if (!pread_all(rs.fd, hdr, sizeof(hdr), 0)) return fail(ARTEA_GPU_EIO, std::string("short read of ") + path);
    if (hdr[0] != kMagic) return fail(ARTEA_GPU_EIO, "bad HGRA magic");
    if (hdr[1] != kVersion) return fail(ARTEA_GPU_EIO, "unsupported HGRA version");
    const uint32_t n = hdr[2], top = hdr[3], ul = hdr[4], bl = hdr[5], entry = hdr[6];
    if (top == kNone || (entry != kNone && entry >= n && n != 0)) return fail(ARTEA_GPU_EIO, "invalid HGRA header");
    if (top >= 64) return fail(ARTEA_GPU_EIO, "HGRA top level above 63 is not supported");
    const uint64_t rec_words = bytes / 4 - 7;
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
    for (int i = 0; i < kReaders; ++i) {
        if (cudaHostAlloc(reinterpret_cast<void**>(&rs.pinned[i]), kChunkWords * 4, cudaHostAllocDefault) !=
                cudaSuccess ||
            cudaEventCreateWithFlags(&rs.copied[i], cudaEventDisableTiming) != cudaSuccess)
            return cleanup(fail(ARTEA_GPU_ENOMEM, "pinned staging buffers unavailable"));
    }
    try {
        // Per vertex: highest level and first row (file order); per row in file
        // order: id count and the raw word of its first id. Arrays that every
        // element of is written before it is read are left uninitialised.
        std::unique_ptr<uint32_t[]> hl(new uint32_t[n]);
        std::unique_ptr<uint64_t[]> vrow(new uint64_t[n]);
        std::vector<uint32_t> rcnt;
        std::vector<uint64_t> rsrc;
        const uint64_t row_cap = std::min<uint64_t>(static_cast<uint64_t>(top + 1) * n, rec_words);
        rcnt.reserve(row_cap);
        rsrc.reserve(row_cap);
        uint64_t gsize[kGroupsMax] = {};
        uint64_t total_ids = 0;
        uint32_t v = 0;        // vertex whose record is being read
        int state = 0;         // 0: a record starts, 1: a count next, 2: skipping a row's ids
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
        const uint64_t nchunks = (rec_words + kChunkWords - 1) / kChunkWords;
        try {
            for (int t = 0; t < kReaders && static_cast<uint64_t>(t) < nchunks; ++t)
                rs.readers.emplace_back(read_chunks, &rs, t, nchunks, rec_words);
        } catch (...) {
            rs.stop_readers();
            return cleanup(fail(ARTEA_GPU_ENOMEM, "cannot start snapshot reader threads"));
        }
        for (uint64_t chunk = 0; chunk < nchunks && err.empty(); ++chunk) {
            const uint64_t off = chunk * kChunkWords;
            const size_t cw = static_cast<size_t>(std::min<uint64_t>(kChunkWords, rec_words - off));
            const int b = static_cast<int>(chunk % kReaders);
            bool read_ok = false;
            {
                std::unique_lock<std::mutex> lk(rs.mu);
                rs.cv.wait(lk, [&] { return rs.holds[b] == chunk; });
                read_ok = rs.read_ok[b];
            }
            if (!read_ok) {
                err = std::string("short read of ") + path;
                break;
            }
            const uint32_t* w = rs.pinned[b];
            CUDA_TRY_IX(cudaMemcpyAsync(rs.d_raw + off, w, cw * 4, cudaMemcpyHostToDevice, rs.stream));
            CUDA_TRY_IX(cudaEventRecord(rs.copied[b], rs.stream));
            size_t i = 0;
            while (i < cw) {
                if (state == 0) {
                    if (v >= n) {
                        err = "HGRA has trailing bytes";
                        break;
                    }
                    const uint32_t h = w[i];
                    if (h == kNone) {
                        hl[v++] = kNone;
                        ++i;
                        continue;
                    }
                    if (h > top) {
                        err = "HGRA vid " + std::to_string(v) + " above top level";
                        break;
                    }
                    hl[v] = h;
                    gsize[h]++;
                    vrow[v] = rcnt.size();
                    // A record that ends inside the chunk is walked row by row;
                    // one that runs past it continues in the word-by-word states.
                    size_t p = i + 1;
                    uint32_t k = 0;
                    for (; k <= h && p < cw; ++k) p += 1 + static_cast<size_t>(w[p]);
                    if (k <= h || p > cw) {
                        lvl = h;
                        state = 1;
                        ++i;
                        continue;
                    }
                    p = i + 1;
                    for (uint32_t l = h;; --l) {
                        const uint32_t cnt = w[p];
                        if (cnt > (l == 0 ? bl : ul)) {
                            err = "HGRA row longer than its level capacity";
                            break;
                        }
                        rcnt.push_back(cnt);
                        rsrc.push_back(off + p + 1);
                        total_ids += cnt;
                        p += 1 + static_cast<size_t>(cnt);
                        if (l == 0) break;
                    }
                    if (!err.empty()) break;
                    i = p;
                    ++v;
                    continue;
                }
                if (state == 2) {
                    const uint64_t k = std::min<uint64_t>(skip, cw - i);
                    i += k;
                    skip -= k;
                    if (skip == 0) row_done();
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
            // The buffer goes back to its reader once its copy has completed.
            CUDA_TRY_IX(cudaEventSynchronize(rs.copied[b]));
            {
                std::lock_guard<std::mutex> lk(rs.mu);
                rs.holds[b] = kFree;
            }
            rs.cv.notify_all();
        }
        rs.stop_readers();
        if (err.empty() && state == 1) err = "HGRA truncated in vid " + std::to_string(v);
        if (err.empty() && v < n) err = "HGRA truncated at vid " + std::to_string(v);
        CUDA_TRY_IX(cudaStreamSynchronize(rs.stream));
        if (!err.empty()) return cleanup(fail(ARTEA_GPU_EIO, err));

        // ---- vertex table and CSR offsets (restore's layout) ----
        const uint32_t groups = top + 1;
        std::unique_ptr<uint32_t[]> vinfo(new uint32_t[2ull * n]);
        uint64_t gstart[kGroupsMax + 1] = {};
        for (uint32_t h = 0; h < groups; ++h) gstart[h + 1] = gstart[h] + gsize[h];
        std::unique_ptr<uint32_t[]> order(new uint32_t[gstart[groups]]);   // vertices by highest level, vid order
        uint64_t fill[kGroupsMax];
        for (uint32_t h = 0; h < groups; ++h) fill[h] = gstart[h];
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
        RowGroups gr;
        std::memset(&gr, 0, sizeof(gr));
        gr.groups = groups;
        uint64_t num_offsets = 0;
        for (uint32_t h = 0; h < groups; ++h) {
            gr.obase[h] = num_offsets;
            num_offsets += gsize[h] * (h + 1ull) + 1;
            gr.row_begin[h + 1] = gr.row_begin[h] + gsize[h] * (h + 1ull);
        }
        const uint64_t num_rows = gr.row_begin[groups];
        std::unique_ptr<uint64_t[]> offs(new uint64_t[num_offsets]);
        std::unique_ptr<unsigned long long[]> csrc(new unsigned long long[std::max<uint64_t>(num_rows, 1)]);
        std::vector<const uint64_t*> gptr(groups);
        {
            uint64_t at = 0, row = 0;
            for (uint32_t h = 0; h < groups; ++h) {
                uint64_t* o = offs.get() + gr.obase[h];
                gptr[h] = o;
                uint64_t rr = 0;
                for (uint64_t k = gstart[h]; k < gstart[h + 1]; ++k) {
                    const uint64_t fr = vrow[order[k]];
                    for (uint32_t j = 0; j <= h; ++j, ++row) {
                        o[rr++] = at;
                        csrc[row] = rsrc[fr + j];
                        at += rcnt[fr + j];
                    }
                }
                o[rr] = at;
            }
        }
        ix->n_offsets = num_offsets;
        ix->n_nbrs = total_ids;
        if (int rc = dev_alloc(&ix->d_vinfo, n)) return cleanup(rc);
        if (int rc = dev_alloc(&ix->d_offsets, num_offsets)) return cleanup(rc);
        if (int rc = dev_alloc(&ix->d_nbrs, std::max<uint64_t>(total_ids, 1))) return cleanup(rc);
        if (int rc = dev_alloc(&rs.d_flags, 1)) return cleanup(rc);
        CUDA_TRY_IX(cudaMemcpy(ix->d_vinfo, vinfo.get(), sizeof(uint2) * n, cudaMemcpyHostToDevice));
        CUDA_TRY_IX(cudaMemcpy(ix->d_offsets, offs.get(), sizeof(uint64_t) * num_offsets, cudaMemcpyHostToDevice));
        CUDA_TRY_IX(cudaMemset(rs.d_flags, 0, sizeof(uint32_t)));
        for (uint32_t h = 0; h < groups; ++h) ix->group_ptr[h] = ix->d_offsets + gr.obase[h];
        if (num_rows) {
            if (int rc = dev_alloc(&rs.d_src, num_rows)) return cleanup(rc);
            CUDA_TRY_IX(cudaMemcpy(rs.d_src, csrc.get(), sizeof(unsigned long long) * num_rows,
                                   cudaMemcpyHostToDevice));
            int sms = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            const uint64_t want = (num_rows + 7) / 8;   // 8 warps per block
            const int grid = static_cast<int>(std::min<uint64_t>(want, static_cast<uint64_t>(std::max(sms, 1)) * 16));
            hgra_rows_kernel<<<grid, 256, 0, rs.stream>>>(rs.d_raw, rs.d_src, gr, ix->d_offsets, ix->d_vinfo, n,
                                                          ix->d_nbrs, rs.d_flags);
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
        if (int rc = index_finish_l0(ix, vinfo.get(), gptr.data())) return cleanup(rc);
    } catch (const std::bad_alloc&) {
        return cleanup(fail(ARTEA_GPU_ENOMEM, "host memory for the snapshot layout unavailable"));
    }
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
