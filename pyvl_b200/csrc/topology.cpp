// Host-side mesh topology for the C ABI: element loops -> unique lines + signed ring CSR,
// dual mesh, element round trip and the line -> ring map.  All O(total entries).
#include <cstdint>
#include <cstring>
#include <vector>

#include "pvl_status.h"

namespace {

inline uint32_t idx_of(uint32_t g) { return g & 0x7FFFFFFFu; }
inline uint32_t rev_of(uint32_t g) { return g >> 31; }

// Open-addressing table of unordered node pairs -> line index.
struct PairTable {
    std::vector<uint32_t> slots;
    uint64_t mask;
    explicit PairTable(size_t n)
    {
        size_t cap = 16;
        while (cap < 2 * n + 16)
            cap <<= 1;
        slots.assign(cap, 0xFFFFFFFFu);
        mask = cap - 1;
    }
    static uint64_t hash(uint32_t a, uint32_t b)
    {
        const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
        uint64_t h = (lo << 32) | hi;
        h ^= h >> 33;
        h *= 0xff51afd7ed558ccdull;
        h ^= h >> 33;
        h *= 0xc4ceb9fe1a85ec53ull;
        h ^= h >> 33;
        return h;
    }
};

}  // namespace

extern "C" int pvl_mesh_from_elements(uint32_t n_points, uint32_t n_elements, const uint32_t* counts,
                                      const uint32_t* flat_points, uint32_t* lines_out,
                                      uint32_t* surface_lines_out, uint32_t* offsets_out,
                                      uint32_t* n_lines_out)
{
    if ((n_elements && (!counts || !flat_points)) || !offsets_out || !n_lines_out)
        return pvl_fail(PVL_ERR_ARG, "pvl_mesh_from_elements: null pointer argument");
    uint64_t total = 0;
    for (uint32_t e = 0; e < n_elements; ++e) {
        if (counts[e] < 3)
            return pvl_fail(PVL_ERR_ARG, "Element %u had only %u indices given (at least 3 are needed).", e,
                            counts[e]);
        total += counts[e];
    }
    if (total > 0x7FFFFFFFull)
        return pvl_fail(PVL_ERR_ARG, "too many element entries (%llu)", (unsigned long long)total);
    // Same bound as the reference (src/meshobject.c:90): ids equal to n_points are accepted.
    uint64_t off = 0;
    for (uint32_t e = 0; e < n_elements; ++e) {
        for (uint32_t k = 0; k < counts[e]; ++k) {
            const uint32_t v = flat_points[off + k];
            if (v > n_points)
                return pvl_fail(PVL_ERR_ARG,
                                "Element %u had specified a point with index %u as its %u point, while only %u "
                                "points were given.",
                                e, v, k, n_points);
        }
        off += counts[e];
    }
    if (total && (!lines_out || !surface_lines_out))
        return pvl_fail(PVL_ERR_ARG, "pvl_mesh_from_elements: null output array");

    PairTable table((size_t)total);
    uint32_t n_lines = 0;
    uint64_t offset = 0;
    offsets_out[0] = 0;
    for (uint32_t e = 0; e < n_elements; ++e) {
        const uint32_t n = counts[e];
        uint32_t left = flat_points[offset + n - 1];
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t right = flat_points[offset + i];
            uint64_t slot = PairTable::hash(left, right) & table.mask;
            uint32_t line = 0xFFFFFFFFu, orient = 0;
            while (table.slots[slot] != 0xFFFFFFFFu) {
                const uint32_t c = table.slots[slot];
                if (lines_out[2 * c] == left && lines_out[2 * c + 1] == right) {
                    line = c;
                    orient = 0;
                    break;
                }
                if (lines_out[2 * c + 1] == left && lines_out[2 * c] == right) {
                    line = c;
                    orient = 1;
                    break;
                }
                slot = (slot + 1) & table.mask;
            }
            if (line == 0xFFFFFFFFu) {
                line = n_lines;
                lines_out[2 * n_lines] = left;
                lines_out[2 * n_lines + 1] = right;
                table.slots[slot] = n_lines;
                n_lines += 1;
            }
            surface_lines_out[offset + i] = (orient << 31) | line;
            left = right;
        }
        offset += n;
        offsets_out[e + 1] = (uint32_t)offset;
    }
    *n_lines_out = n_lines;
    return PVL_OK;
}

extern "C" int pvl_mesh_dual(uint32_t n_points, uint32_t n_lines, const uint32_t* lines, uint32_t n_surfaces,
                             const uint32_t* surface_offsets, const uint32_t* surface_lines,
                             uint32_t* dual_lines_out, uint32_t* dual_offsets_out, uint32_t* dual_surface_lines_out)
{
    if (!surface_offsets || (n_lines && (!lines || !dual_lines_out || !dual_surface_lines_out)) || !dual_offsets_out)
        return pvl_fail(PVL_ERR_ARG, "pvl_mesh_dual: null pointer argument");
    // Dual lines: the first two rings (in ring order) that hold each line; a ring counts
    // once per line (src/core/mesh.c:88-111).
    std::vector<uint32_t> cnt(n_lines, 0), last_ring(n_lines, 0xFFFFFFFFu);
    for (uint32_t i = 0; i < n_lines; ++i) {
        dual_lines_out[2 * i] = PVL_INVALID_ID;
        dual_lines_out[2 * i + 1] = PVL_INVALID_ID;
    }
    for (uint32_t s = 0; s < n_surfaces; ++s) {
        for (uint32_t k = surface_offsets[s]; k < surface_offsets[s + 1]; ++k) {
            const uint32_t g = surface_lines[k];
            const uint32_t l = idx_of(g);
            if (l >= n_lines)
                return pvl_fail(PVL_ERR_TOPOLOGY, "surface %u references line %u of %u", s, l, n_lines);
            if (last_ring[l] == s)
                continue;
            last_ring[l] = s;
            if (cnt[l] < 2) {
                dual_lines_out[2 * l + (rev_of(g) ? 0 : 1)] = s;
                cnt[l] += 1;
            }
        }
    }
    // Dual surfaces: lines touching each point, in line order, p1 before p2 (mesh.c:118-169).
    std::vector<uint32_t> deg(n_points + 1, 0);
    for (uint32_t i = 0; i < n_lines; ++i) {
        if (lines[2 * i] < n_points)
            deg[lines[2 * i]] += 1;
        if (lines[2 * i + 1] < n_points)
            deg[lines[2 * i + 1]] += 1;
    }
    dual_offsets_out[0] = 0;
    for (uint32_t p = 0; p < n_points; ++p)
        dual_offsets_out[p + 1] = dual_offsets_out[p] + deg[p];
    std::vector<uint32_t> fill(dual_offsets_out, dual_offsets_out + n_points);
    for (uint32_t i = 0; i < n_lines; ++i) {
        const uint32_t a = lines[2 * i], b = lines[2 * i + 1];
        if (a < n_points)
            dual_surface_lines_out[fill[a]++] = i;
        if (b < n_points)
            dual_surface_lines_out[fill[b]++] = i | 0x80000000u;
    }
    return PVL_OK;
}

extern "C" int pvl_mesh_to_elements(uint32_t n_surfaces, const uint32_t* surface_offsets,
                                    const uint32_t* surface_lines, const uint32_t* lines, uint32_t* counts_out,
                                    uint32_t* flat_out)
{
    if (!surface_offsets || (n_surfaces && (!counts_out || !flat_out || !surface_lines || !lines)))
        return pvl_fail(PVL_ERR_ARG, "pvl_mesh_to_elements: null pointer argument");
    // src/core/mesh.c:262-295: a reversed line contributes its first point, a forward one its last.
    for (uint32_t s = 0; s < n_surfaces; ++s) {
        counts_out[s] = surface_offsets[s + 1] - surface_offsets[s];
        for (uint32_t k = surface_offsets[s]; k < surface_offsets[s + 1]; ++k) {
            const uint32_t g = surface_lines[k];
            flat_out[k] = rev_of(g) ? lines[2 * idx_of(g)] : lines[2 * idx_of(g) + 1];
        }
    }
    return PVL_OK;
}

extern "C" int pvl_line_ring_map(uint32_t n_lines, uint32_t n_surfaces, const uint32_t* surface_offsets,
                                 const uint32_t* surface_lines, uint32_t* map_offsets_out, uint32_t* map_entries_out)
{
    if (!surface_offsets || !map_offsets_out)
        return pvl_fail(PVL_ERR_ARG, "pvl_line_ring_map: null pointer argument");
    std::vector<uint32_t> deg(n_lines, 0);
    for (uint32_t s = 0; s < n_surfaces; ++s)
        for (uint32_t k = surface_offsets[s]; k < surface_offsets[s + 1]; ++k) {
            const uint32_t l = idx_of(surface_lines[k]);
            if (l >= n_lines)
                return pvl_fail(PVL_ERR_TOPOLOGY, "surface %u references line %u of %u", s, l, n_lines);
            deg[l] += 1;
        }
    map_offsets_out[0] = 0;
    for (uint32_t l = 0; l < n_lines; ++l)
        map_offsets_out[l + 1] = map_offsets_out[l] + deg[l];
    std::vector<uint32_t> fill(map_offsets_out, map_offsets_out + n_lines);
    for (uint32_t s = 0; s < n_surfaces; ++s)
        for (uint32_t k = surface_offsets[s]; k < surface_offsets[s + 1]; ++k) {
            const uint32_t g = surface_lines[k];
            map_entries_out[fill[idx_of(g)]++] = s | (g & 0x80000000u);
        }
    return PVL_OK;
}
