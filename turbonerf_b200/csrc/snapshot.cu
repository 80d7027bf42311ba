// .turbo snapshots of a trained NeRF, in the reference's file layout (FileManager::save / load,
// src/services/file-manager.cuh:18-198): a 300-byte header (project name "TurboNeRF", dataset
// path, version 0, parameter counts, bitfield size, AABB scale, appearance count), the fp32
// parameters, then the occupancy bitfield. This library appends a resume block that the
// reference's loader never reads (it stops after the bitfield): magic "TNRESUME", the cascade
// and parameter layout, the step counters, then Adam's first and second moments and per-parameter
// step counts and the grid densities, so that training continues exactly where it stopped.
#include <cstdio>
#include <cstring>

#include "tn_internal.cuh"

namespace tn {

int read_turbo_file(const char* path, TurboHeader* header, TurboResume* resume, bool* has_resume, uint64_t* size) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(TN_E_INVALID, "cannot open %s", path);
    TurboHeader h{};
    const bool got = std::fread(&h, sizeof(h), 1, f) == 1;
    std::fseek(f, 0, SEEK_END);
    const long end = std::ftell(f);
    int st = TN_OK;
    if (!got || std::strncmp(h.project_name, "TurboNeRF", sizeof(h.project_name)) != 0) {
        st = fail(TN_E_INVALID, "%s is not a TurboNeRF file", path);
    } else if (h.version != 0) {
        st = fail(TN_E_INVALID, "%s: file version %u is not supported (0 is)", path, h.version);
    } else {
        const uint64_t n_params = (uint64_t)h.n_color_params + h.n_density_params + h.n_appearance_embedding_params;
        const uint64_t body = sizeof(TurboHeader) + 4 * n_params + h.n_occ_grid_bits;
        if ((uint64_t)end < body) {
            st = fail(TN_E_INVALID, "%s: truncated (%ld bytes, the sections need %llu)", path, end,
                      (unsigned long long)body);
        } else {
            TurboResume r{};
            bool has = false;
            if ((uint64_t)end >= body + sizeof(TurboResume)) {
                std::fseek(f, (long)body, SEEK_SET);
                has = std::fread(&r, sizeof(r), 1, f) == 1 && std::memcmp(r.magic, "TNRESUME", 8) == 0;
            }
            if (has && r.version != 1) st = fail(TN_E_INVALID, "%s: resume block version %u is not supported", path, r.version);
            if (resume) *resume = r;
            if (has_resume) *has_resume = has;
        }
    }
    std::fclose(f);
    if (header) *header = h;
    if (size) *size = end < 0 ? 0 : (uint64_t)end;
    return st;
}

}  // namespace tn

using namespace tn;

extern "C" {

int tn_turbo_file_info(const char* path, tn_turbo_info* out) {
    TN_NONNULL(path); TN_NONNULL(out);
    TurboHeader h;
    TurboResume r;
    bool has = false;
    uint64_t size = 0;
    const int st = read_turbo_file(path, &h, &r, &has, &size);
    if (st != TN_OK) return st;
    *out = tn_turbo_info{};
    out->n_params = (uint64_t)h.n_color_params + h.n_density_params + h.n_appearance_embedding_params;
    out->n_occ_grid_bits = h.n_occ_grid_bits;
    out->aabb_scale = h.aabb_scale;
    out->has_resume = has ? 1u : 0u;
    out->step_count = has ? r.step_count : 0u;
    out->n_levels = has ? r.n_levels : 0u;
    out->resolution = has ? r.resolution : 0u;
    out->file_bytes = size;
    std::memcpy(out->dataset_path, h.dataset_path, sizeof(out->dataset_path));
    out->dataset_path[sizeof(out->dataset_path) - 1] = '\0';
    return TN_OK;
}

}  // extern "C"
