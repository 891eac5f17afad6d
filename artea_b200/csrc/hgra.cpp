// HGRA v1 snapshots and host-side graph validation (no GPU needed).
//
// Wire format (index/persistence/hierarchical_graph_file_manager.hpp:15-39):
//   header: 7 x uint32 (magic 'HGRA' = 0x48475241, version 1, num_vertices,
//           top_level_id, ul_max_nbr_size, bl_max_nbr_size, entry_point_vid)
//   per vid: highest_level_id; if not 0xFFFFFFFF, for level = highest..0:
//            count, then count neighbour ids.
// Restore (hierarchical_graph_file_manager.hpp:152-300) buckets vids by highest
// level in vid order (local_vid = rank within its bucket) and lays the CSR out
// group by group, each vertex's rows from its highest level down to 0. The
// reader below produces the same layout and applies the same checks.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/artea_gpu.h"
#include "common.h"

namespace {

constexpr uint32_t kMagic = 0x48475241u;
constexpr uint32_t kVersion = 1u;
constexpr uint32_t kInvalid = 0xffffffffu;

struct Reader {
    std::vector<uint32_t> words;
    size_t pos = 0;
    bool take(uint32_t& v) {
        if (pos >= words.size()) return false;
        v = words[pos++];
        return true;
    }
};

int load_words(const char* path, Reader& r) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return artea_gpu::fail(ARTEA_GPU_EIO, std::string("cannot open ") + path);
    std::fseek(fp, 0, SEEK_END);
    const long bytes = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    if (bytes < 28 || bytes % 4 != 0) {
        std::fclose(fp);
        return artea_gpu::fail(ARTEA_GPU_EIO, std::string("truncated or misaligned snapshot ") + path);
    }
    r.words.resize(static_cast<size_t>(bytes) / 4);
    const size_t got = std::fread(r.words.data(), 4, r.words.size(), fp);
    std::fclose(fp);
    if (got != r.words.size()) return artea_gpu::fail(ARTEA_GPU_EIO, std::string("short read of ") + path);
    return ARTEA_GPU_OK;
}

// Parses the whole snapshot; fills info and, when the output pointers are set,
// the CSR arrays.
int parse(const char* path, artea_gpu_hgra_info* info, uint32_t* vinfo, uint64_t* offsets, uint32_t* nbrs) {
    Reader r;
    if (int rc = load_words(path, r)) return rc;
    uint32_t hdr[7];
    for (auto& h : hdr) r.take(h);
    if (hdr[0] != kMagic) return artea_gpu::fail(ARTEA_GPU_EIO, "bad HGRA magic");
    if (hdr[1] != kVersion) return artea_gpu::fail(ARTEA_GPU_EIO, "unsupported HGRA version");
    const uint32_t n = hdr[2], top = hdr[3], ul = hdr[4], bl = hdr[5], entry = hdr[6];
    if (top == kInvalid || (entry != kInvalid && entry >= n && n != 0))
        return artea_gpu::fail(ARTEA_GPU_EIO, "invalid HGRA header");
    if (top >= 64) return artea_gpu::fail(ARTEA_GPU_EIO, "HGRA top level above 63 is not supported");
    const uint32_t groups = top + 1;

    std::vector<uint32_t> hl(n);
    std::vector<size_t> rec(n);        // word position of each vid's first count
    std::vector<uint64_t> gsize(groups, 0);
    uint64_t total_ids = 0;
    for (uint32_t v = 0; v < n; ++v) {
        uint32_t h;
        if (!r.take(h)) return artea_gpu::fail(ARTEA_GPU_EIO, "HGRA truncated at vid " + std::to_string(v));
        hl[v] = h;
        rec[v] = r.pos;
        if (h == kInvalid) continue;
        if (h > top) return artea_gpu::fail(ARTEA_GPU_EIO, "HGRA vid " + std::to_string(v) + " above top level");
        gsize[h]++;
        for (uint32_t lvl = h;; --lvl) {
            uint32_t cnt;
            if (!r.take(cnt)) return artea_gpu::fail(ARTEA_GPU_EIO, "HGRA truncated in vid " + std::to_string(v));
            const uint32_t capacity = lvl == 0 ? bl : ul;
            if (cnt > capacity) return artea_gpu::fail(ARTEA_GPU_EIO, "HGRA row longer than its level capacity");
            if (r.pos + cnt > r.words.size()) return artea_gpu::fail(ARTEA_GPU_EIO, "HGRA truncated in a row");
            for (uint32_t i = 0; i < cnt; ++i)
                if (r.words[r.pos + i] >= n) return artea_gpu::fail(ARTEA_GPU_EIO, "HGRA neighbour id out of range");
            r.pos += cnt;
            total_ids += cnt;
            if (lvl == 0) break;
        }
    }
    if (r.pos != r.words.size()) return artea_gpu::fail(ARTEA_GPU_EIO, "HGRA has trailing bytes");

    info->num_vertices = n;
    info->top_level = top;
    info->ul_max_nbr_size = ul;
    info->bl_max_nbr_size = bl;
    info->entry_point_vid = entry;
    info->num_groups = groups;
    info->num_neighbor_ids = total_ids;
    uint64_t num_offsets = 0;
    for (uint32_t h = 0; h < 64; ++h) info->group_sizes[h] = h < groups ? gsize[h] : 0;
    for (uint32_t h = 0; h < groups; ++h) num_offsets += gsize[h] * (h + 1ull) + 1;
    info->num_offsets = num_offsets;
    if (!vinfo) return ARTEA_GPU_OK;

    // Bucket vids by highest level in vid order.
    std::vector<std::vector<uint32_t>> bucket(groups);
    for (uint32_t h = 0; h < groups; ++h) bucket[h].reserve(gsize[h]);
    for (uint32_t v = 0; v < n; ++v) {
        if (hl[v] == kInvalid) {
            vinfo[2 * v] = kInvalid;
            vinfo[2 * v + 1] = kInvalid;
            continue;
        }
        vinfo[2 * v] = hl[v];
        vinfo[2 * v + 1] = static_cast<uint32_t>(bucket[hl[v]].size());
        bucket[hl[v]].push_back(v);
    }
    uint64_t at = 0;    // running neighbour position
    uint64_t obase = 0; // running offset-array position
    for (uint32_t h = 0; h < groups; ++h) {
        uint64_t* off = offsets + obase;
        uint64_t row = 0;
        for (uint32_t v : bucket[h]) {
            size_t p = rec[v];
            for (uint32_t lvl = h;; --lvl) {
                const uint32_t cnt = r.words[p++];
                off[row++] = at;
                std::memcpy(nbrs + at, &r.words[p], sizeof(uint32_t) * cnt);
                at += cnt;
                p += cnt;
                if (lvl == 0) break;
            }
        }
        off[row] = at;
        obase += gsize[h] * (h + 1ull) + 1;
    }
    return ARTEA_GPU_OK;
}

}  // namespace

extern "C" int artea_gpu_hgra_probe(const char* path, artea_gpu_hgra_info* info) {
    if (!path || !info) return artea_gpu::fail(ARTEA_GPU_EINVAL, "null argument");
    return parse(path, info, nullptr, nullptr, nullptr);
}

extern "C" int artea_gpu_hgra_read(const char* path, uint32_t* vinfo, uint64_t* offsets, uint32_t* nbrs) {
    if (!path || !vinfo || !offsets || !nbrs) return artea_gpu::fail(ARTEA_GPU_EINVAL, "null argument");
    artea_gpu_hgra_info info;
    return parse(path, &info, vinfo, offsets, nbrs);
}

extern "C" int artea_gpu_hgra_write(const char* path, const artea_gpu_graph_desc* g) {
    if (!path || !g) return artea_gpu::fail(ARTEA_GPU_EINVAL, "null argument");
    if (int rc = artea_gpu_graph_validate(g)) return rc;
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return artea_gpu::fail(ARTEA_GPU_EIO, std::string("cannot create ") + path);
    const bool empty = g->num_vertices == 0 || g->top_level == kInvalid;
    const uint32_t hdr[7] = {kMagic, kVersion, g->num_vertices, empty ? 0u : g->top_level,
                             g->ul_max_nbr_size, g->bl_max_nbr_size, g->entry_point_vid};
    bool ok = std::fwrite(hdr, 4, 7, fp) == 7;
    for (uint32_t v = 0; ok && v < g->num_vertices; ++v) {
        const uint32_t h = g->vertex_info[2 * v];
        ok = std::fwrite(&h, 4, 1, fp) == 1;
        if (h == kInvalid) continue;
        const uint64_t local = g->vertex_info[2 * v + 1];
        const uint64_t* off = g->group_offsets[h];
        for (uint32_t lvl = h; ok; --lvl) {
            const uint64_t row = local * (h + 1ull) + (h - lvl);
            const uint32_t cnt = static_cast<uint32_t>(off[row + 1] - off[row]);
            ok = std::fwrite(&cnt, 4, 1, fp) == 1 &&
                 (cnt == 0 || std::fwrite(g->neighbor_ids + off[row], 4, cnt, fp) == cnt);
            if (lvl == 0) break;
        }
    }
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? ARTEA_GPU_OK : artea_gpu::fail(ARTEA_GPU_EIO, std::string("write failed: ") + path);
}

// Host validation before upload: every id the kernels will follow must be in
// range and present on the level of the row that names it, so that no device
// access can leave its buffer.
extern "C" int artea_gpu_graph_validate(const artea_gpu_graph_desc* g) {
    using artea_gpu::fail;
    if (!g) return fail(ARTEA_GPU_EINVAL, "null graph");
    const uint32_t n = g->num_vertices;
    if (n == 0 || g->top_level == kInvalid) return ARTEA_GPU_OK;
    if (g->top_level >= 64) return fail(ARTEA_GPU_EGRAPH, "top level above 63 is not supported");
    if (!g->vertex_info || !g->group_offsets || !g->group_sizes || (g->num_neighbor_ids && !g->neighbor_ids))
        return fail(ARTEA_GPU_EINVAL, "null graph array");
    const uint32_t groups = g->top_level + 1;
    if (g->entry_point_vid >= n) return fail(ARTEA_GPU_EGRAPH, "entry point out of range");
    if (g->vertex_info[2 * g->entry_point_vid] != g->top_level)
        return fail(ARTEA_GPU_EGRAPH, "entry point is not on the top level");
    std::vector<uint64_t> seen(groups, 0);
    for (uint32_t v = 0; v < n; ++v) {
        const uint32_t h = g->vertex_info[2 * v], local = g->vertex_info[2 * v + 1];
        if (h == kInvalid) continue;
        if (h >= groups) return fail(ARTEA_GPU_EGRAPH, "vertex " + std::to_string(v) + " above top level");
        if (local >= g->group_sizes[h]) return fail(ARTEA_GPU_EGRAPH, "vertex " + std::to_string(v) + " local id out of range");
        seen[h]++;
    }
    for (uint32_t h = 0; h < groups; ++h) {
        if (seen[h] != g->group_sizes[h]) return fail(ARTEA_GPU_EGRAPH, "group size does not match vertex table");
        const uint64_t* off = g->group_offsets[h];
        const uint64_t rows = g->group_sizes[h] * (h + 1ull);
        if (!off) return fail(ARTEA_GPU_EINVAL, "null group offsets");
        for (uint64_t rrow = 0; rrow < rows; ++rrow) {
            if (off[rrow + 1] < off[rrow] || off[rrow + 1] > g->num_neighbor_ids)
                return fail(ARTEA_GPU_EGRAPH, "CSR offsets not monotone or past the neighbour array");
            const uint32_t lvl = h - static_cast<uint32_t>(rrow % (h + 1ull));
            const uint64_t len = off[rrow + 1] - off[rrow];
            const uint32_t capacity = lvl == 0 ? g->bl_max_nbr_size : g->ul_max_nbr_size;
            if (len > capacity) return fail(ARTEA_GPU_EGRAPH, "row longer than its level capacity");
            for (uint64_t i = off[rrow]; i < off[rrow + 1]; ++i) {
                const uint32_t id = g->neighbor_ids[i];
                if (id >= n) return fail(ARTEA_GPU_EGRAPH, "neighbour id " + std::to_string(id) + " out of range");
                const uint32_t idh = g->vertex_info[2 * id];
                if (idh == kInvalid || idh < lvl)
                    return fail(ARTEA_GPU_EGRAPH, "neighbour " + std::to_string(id) + " is not on level " +
                                                      std::to_string(lvl));
            }
        }
    }
    return ARTEA_GPU_OK;
}
