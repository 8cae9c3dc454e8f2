// Binary snapshot output from device state: the reference's field and cell
// dumps (crates/marl-output/src/binary_dump.rs:109-120), its ruleset sidecars
// (binary_dump.rs:121-350) and run_meta.json (binary_dump.rs:362-415,
// crates/marl-format/src/lib.rs:130-218), uncompressed.
//
// The field dump is the field buffer itself ([z][y][x][12] f32, the
// reference's Field::data order).  The cell dump is one packed 25-byte
// ViewerCellRecord per cell in cell-vector order (marl-format lib.rs:351-364:
// pos as 3 x f32, lineage_id u64, starter_type u8, energy f32, little
// endian), packed on the device from the cell table so that 25 bytes per
// cell cross to the host instead of the 656-byte record.
#include <cuda_runtime.h>

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "ctx_impl.h"

using namespace marl;

namespace marl {

constexpr uint32_t kViewerStride = 25;

__global__ void k_pack_viewer_cells(CellTable t, uint32_t n, uint8_t* __restrict__ out) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t P = t.pos[j];
    const float pos[3] = {(float)pos_x(P), (float)pos_y(P), (float)pos_z(P)};
    const uint64_t lineage = t.lineage[j];
    const uint8_t starter = (uint8_t)(t.state[j] >> 24);
    const float energy = t.internal[j];
    uint8_t rec[kViewerStride];
    memcpy(rec, pos, 12);
    memcpy(rec + 12, &lineage, 8);
    rec[20] = starter;
    memcpy(rec + 21, &energy, 4);
    uint8_t* dst = out + (size_t)j * kViewerStride;
#pragma unroll
    for (int i = 0; i < (int)kViewerStride; ++i) dst[i] = rec[i];
}

// ---------------------------------------------------------- rulesets -----
// Layer averages: 110 float fields per ruleset (marl-format ruleset_layer_value_count(8, 8, 16, 8)),
// one 448-byte record per z layer.
constexpr int kLayerValues = 3 * MARL_S_RECEPTORS + 2 * MARL_S_TRANSPORTERS + 3 * MARL_R_MAX + 2 * MARL_S_EFFECTORS + 6;
constexpr int kLayerStride = 8 + 4 * kLayerValues;
static_assert(kLayerValues == 110 && kLayerStride == 448, "ruleset layer record");
constexpr int kCanonicalBytes = 536;     // canonical ruleset payload (marl-format lib.rs:70-89)
constexpr int kCanonicalRecord = 544;    // + x, y, z u16 and 2 pad bytes, as the device packs it
constexpr int kLayerThreads = 128;
constexpr uint32_t kLayerChunk = 2048;

// Field v (0..109) of cell j's ruleset, in the order binary_dump.rs:121-150
// accumulates them.
__device__ __forceinline__ float layer_value(const CellTable& t, uint32_t j, int v) {
    const size_t cap = t.cap;
    if (v < 24) return t.cold[(size_t)j * kColdFloats + v];  // receptors: k_half, n_hill, gain
    v -= 24;
    if (v < 16) {
        const float2 r = t.tp_rate[(size_t)(v >> 1) * cap + j];
        return (v & 1) ? r.y : r.x;
    }
    v -= 16;
    if (v < 48) {
        const uint4 q = t.rx[(size_t)(v / 3) * cap + j];
        const int h = v % 3;
        return __uint_as_float(h == 0 ? q.y : (h == 1 ? q.z : q.w));  // k_m, v_max, k_cat
    }
    v -= 48;
    if (v < 16) {
        const float2 p = t.ef_par[(size_t)(v >> 1) * cap + j];
        return (v & 1) ? p.y : p.x;  // threshold, rate
    }
    v -= 16;
    if (v < 4) {
        const float4 f = t.fate[j];
        return v == 0 ? f.x : (v == 1 ? f.y : (v == 2 ? f.z : f.w));
    }
    return t.cold[(size_t)j * kColdFloats + 24 + (v - 4)];  // hgt_propensity, mutation_rate
}

// Block z: the sums of the 110 fields over the cells of layer z, in cell
// order (thread v owns field v), as f64; then the f32 averages.
__global__ void __launch_bounds__(kLayerThreads) k_ruleset_layers(CellTable t, uint32_t n, uint8_t* __restrict__ out) {
    __shared__ uint32_t s_pos[kLayerChunk];
    const uint32_t z = blockIdx.x;
    const int v = threadIdx.x;
    double sum = 0.0;
    uint32_t count = 0;
    for (uint32_t base = 0; base < n; base += kLayerChunk) {
        const uint32_t m = n - base < kLayerChunk ? n - base : kLayerChunk;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < m; i += kLayerThreads) s_pos[i] = t.pos[base + i];
        __syncthreads();
        for (uint32_t i = 0; i < m; ++i) {
            if (pos_z(s_pos[i]) != z) continue;  // uniform across the block
            ++count;
            if (v < kLayerValues) sum += (double)layer_value(t, base + i, v);
        }
    }
    uint8_t* rec = out + (size_t)z * kLayerStride;
    if (threadIdx.x == 0) {
        const uint16_t zz = (uint16_t)z, zero = 0;
        memcpy(rec, &zz, 2);
        memcpy(rec + 2, &zero, 2);
        memcpy(rec + 4, &count, 4);
    }
    if (v < kLayerValues) {
        const float avg = count > 0 ? (float)(sum / (double)count) : 0.0f;
        memcpy(rec + 8 + 4 * v, &avg, 4);
    }
}

struct ByteWriter {
    uint8_t* p;
    __device__ void f32(float v) {
        const uint32_t b = __float_as_uint(v);
        p[0] = (uint8_t)b, p[1] = (uint8_t)(b >> 8), p[2] = (uint8_t)(b >> 16), p[3] = (uint8_t)(b >> 24);
        p += 4;
    }
    __device__ void u8(uint32_t v) { *p++ = (uint8_t)v; }
};

// Cell j's canonical 536-byte ruleset followed by x, y, z (u16) and 2 zero
// bytes: one 544-byte record per cell.
__global__ void k_ruleset_canonical(CellTable t, uint32_t n, uint8_t* __restrict__ out) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const size_t cap = t.cap;
    ByteWriter w{out + (size_t)j * kCanonicalRecord};
    const float* cold = t.cold + (size_t)j * kColdFloats;
    for (int i = 0; i < 3 * MARL_S_RECEPTORS; ++i) w.f32(cold[i]);
    const uint4 tpi = t.tp_idx[j];
    const uint32_t tw[4] = {tpi.x, tpi.y, tpi.z, tpi.w};
    for (int i = 0; i < MARL_S_TRANSPORTERS; ++i) {
        const float2 r = t.tp_rate[(size_t)i * cap + j];
        const uint32_t pair = (tw[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;  // ext | int << 8
        w.f32(r.x), w.f32(r.y), w.u8(pair & 0xFF), w.u8(pair >> 8);
    }
    for (int r = 0; r < MARL_R_MAX; ++r) {
        const uint4 q = t.rx[(size_t)r * cap + j];
        w.u8(q.x & 0xFF), w.u8((q.x >> 8) & 0xFF), w.u8((q.x >> 16) & 0xFF), w.u8(q.x >> 24);
        w.f32(__uint_as_float(q.y)), w.f32(__uint_as_float(q.z)), w.f32(__uint_as_float(q.w));
    }
    const uint4 efi = t.ef_idx[j];
    const uint32_t ew[4] = {efi.x, efi.y, efi.z, efi.w};
    for (int i = 0; i < MARL_S_EFFECTORS; ++i) {
        const float2 p = t.ef_par[(size_t)i * cap + j];
        const uint32_t pair = (ew[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;  // int | ext << 8
        w.f32(p.x), w.f32(p.y), w.u8(pair & 0xFF), w.u8(pair >> 8);
    }
    const float4 f = t.fate[j];
    w.f32(f.x), w.f32(f.y), w.f32(f.z), w.f32(f.w);
    w.f32(cold[24]), w.f32(cold[25]);
    const uint32_t P = t.pos[j];
    const uint32_t xyz[3] = {pos_x(P), pos_y(P), pos_z(P)};
    for (int k = 0; k < 3; ++k) w.u8(xyz[k] & 0xFF), w.u8(xyz[k] >> 8);
    w.u8(0), w.u8(0);
}

static bool write_file(const std::string& path, const void* data, size_t bytes) {
    const std::string tmp = path + ".tmp";  // written whole, then renamed (binary_dump.rs:76-100)
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(data, 1, bytes, f) == bytes;
    if (std::fclose(f) != 0 || !ok) {
        std::remove(tmp.c_str());
        return false;
    }
    return std::rename(tmp.c_str(), path.c_str()) == 0;
}

static const char* ruleset_mode_name(int mode) {
    switch (mode) {
        case MARL_RULESETS_LAYERS: return "layer_averages";
        case MARL_RULESETS_FULL: return "full";
        case MARL_RULESETS_BOTH: return "both";
        default: return "off";
    }
}

// run_meta.json with the keys of binary_dump.rs:362-415 that describe this
// library's files (the payload-layout prose strings are left out).
static bool write_run_meta(const std::string& dir, int gx, int gy, int gz, bool field, bool cells, int ruleset_mode) {
    const uint64_t field_count = (uint64_t)gx * gy * gz * MARL_S_EXT;
    std::string m;
    char buf[1536];
    std::snprintf(buf, sizeof(buf),
                  "{\n  \"grid_x\": %d,\n  \"grid_y\": %d,\n  \"grid_z\": %d,\n  \"s_ext\": %d,\n  \"m_int\": %d,\n"
                  "  \"field_dtype\": \"f32\",\n  \"field_layout\": \"z_y_x_species\",\n"
                  "  \"field_byte_len\": %llu,\n  \"cell_record_stride\": %u,\n  \"endianness\": \"little\",\n"
                  "  \"binary_format_version\": 2,\n  \"binary_compression\": \"none\",\n"
                  "  \"binary_compression_level\": 0,\n  \"write_binary_field\": %s,\n  \"write_binary_cells\": %s,\n"
                  "  \"field_file_pattern\": \"tick_<T>.field.bin\",\n  \"cell_file_pattern\": \"tick_<T>.cells.bin\",\n"
                  "  \"field_count\": %llu,\n  \"cell_header_byte_len\": 0,\n"
                  "  \"cell_count_source\": \"file_size_divided_by_cell_record_stride\",\n"
                  "  \"cell_pos_units\": \"grid_voxel_indices\",\n"
                  "  \"cell_record_layout\": \"pos:f32[3],lineage_id:u64,starter_type:u8,energy:f32\",\n"
                  "  \"ruleset_output_mode\": \"%s\",\n"
                  "  \"ruleset_layer_file_pattern\": \"tick_<T>.ruleset_layers.bin\",\n"
                  "  \"ruleset_layer_record_stride\": %d",
                  gx, gy, gz, MARL_S_EXT, MARL_M_INT, (unsigned long long)(field_count * 4), kViewerStride,
                  field ? "true" : "false", cells ? "true" : "false", (unsigned long long)field_count,
                  ruleset_mode_name(ruleset_mode), kLayerStride);
    m = buf;
    if (ruleset_mode & MARL_RULESETS_FULL) {
        std::snprintf(buf, sizeof(buf),
                      ",\n  \"ruleset_full_file_pattern\": \"tick_<T>.rulesets.bin\",\n"
                      "  \"ruleset_full_header_size\": 24,\n  \"ruleset_full_ruleset_byte_size\": %d,\n"
                      "  \"ruleset_full_cell_ref_stride\": 10,\n  \"ruleset_full_magic_ascii\": \"MRSF\",\n"
                      "  \"ruleset_full_format_version\": 1",
                      kCanonicalBytes);
        m += buf;
    }
    m += "\n}\n";
    return write_file(dir + "/run_meta.json", m.data(), m.size());
}

// The MRSF v1 file from per-cell 544-byte records (canonical ruleset + x, y,
// z): distinct rulesets in order of first occurrence (binary_dump.rs:272-350).
static std::vector<uint8_t> assemble_full_dump(const uint8_t* recs, uint32_t n) {
    std::unordered_map<std::string, uint32_t> dict;
    dict.reserve(n);
    std::vector<uint32_t> ids(n);
    std::vector<const uint8_t*> entries;
    for (uint32_t j = 0; j < n; ++j) {
        const uint8_t* r = recs + (size_t)j * kCanonicalRecord;
        auto it = dict.emplace(std::string(reinterpret_cast<const char*>(r), kCanonicalBytes), (uint32_t)entries.size());
        if (it.second) entries.push_back(r);
        ids[j] = it.first->second;
    }
    const uint32_t dict_count = (uint32_t)entries.size();
    std::vector<uint8_t> out;
    out.reserve(24 + (size_t)dict_count * kCanonicalBytes + (size_t)n * 10);
    auto put32 = [&](uint32_t v) {
        for (int k = 0; k < 4; ++k) out.push_back((uint8_t)(v >> (8 * k)));
    };
    out.insert(out.end(), {'M', 'R', 'S', 'F'});
    put32(1);  // format version
    put32(0);  // flags
    put32(dict_count);
    put32(n);
    put32(kCanonicalBytes);
    for (const uint8_t* e : entries) out.insert(out.end(), e, e + kCanonicalBytes);
    for (uint32_t j = 0; j < n; ++j) {
        const uint8_t* r = recs + (size_t)j * kCanonicalRecord + kCanonicalBytes;
        out.insert(out.end(), r, r + 6);  // x, y, z u16
        put32(ids[j]);
    }
    return out;
}

static marl_status write_ruleset_files(const std::string& dir, uint64_t tick, const Grid& g, int mode,
                                       const uint8_t* layers, const uint8_t* canon, uint32_t n) {
    const std::string stem = dir + "/tick_" + std::to_string((unsigned long long)tick);
    if ((mode & MARL_RULESETS_LAYERS) && !write_file(stem + ".ruleset_layers.bin", layers, (size_t)g.Z * kLayerStride))
        return fail(MARL_ERR_INVALID_INPUT, "cannot write %s.ruleset_layers.bin: %s", stem.c_str(), std::strerror(errno));
    if (mode & MARL_RULESETS_FULL) {
        const std::vector<uint8_t> full = assemble_full_dump(canon, n);
        if (!write_file(stem + ".rulesets.bin", full.data(), full.size()))
            return fail(MARL_ERR_INVALID_INPUT, "cannot write %s.rulesets.bin: %s", stem.c_str(), std::strerror(errno));
    }
    if (!write_run_meta(dir, g.X, g.Y, g.Z, true, true, mode))
        return fail(MARL_ERR_INVALID_INPUT, "cannot write %s/run_meta.json: %s", dir.c_str(), std::strerror(errno));
    return MARL_OK;
}

}  // namespace marl

extern "C" {

marl_status marl_ctx_viewer_cells(marl_ctx* c, uint8_t* out, uint64_t cap_bytes, uint32_t* n_out) {
    if (!c || !n_out || (cap_bytes && !out)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    *n_out = c->n;
    const uint64_t bytes = (uint64_t)c->n * kViewerStride;
    if (bytes > cap_bytes) return fail(MARL_ERR_CAPACITY, "%u cells need %llu bytes", c->n, (unsigned long long)bytes);
    if (c->n == 0) return MARL_OK;
    uint8_t* d = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&d, bytes, c->stream);
    if (e == cudaSuccess) {
        k_pack_viewer_cells<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->t, c->n, d);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, c->stream);
        cudaFreeAsync(d, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    }
    if (e != cudaSuccess) return cuda_fail(e, "marl_ctx_viewer_cells");
    c->d2h_bytes += bytes;
    return MARL_OK;
}

marl_status marl_write_dump(const char* dir, uint64_t tick, int32_t gx, int32_t gy, int32_t gz, const float* field,
                            const uint8_t* viewer_cells, uint32_t n_cells) {
    if (!dir || (!field && !viewer_cells)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    marl_status st = validate_dims(gx, gy, gz);
    if (st) return st;
    const std::string base(dir);
    const uint64_t field_bytes = (uint64_t)gx * gy * gz * MARL_S_EXT * 4;
    if (!write_run_meta(base, gx, gy, gz, field != nullptr, viewer_cells != nullptr, 0))
        return fail(MARL_ERR_INVALID_INPUT, "cannot write %s/run_meta.json: %s", base.c_str(), std::strerror(errno));
    const std::string stem = base + "/tick_" + std::to_string((unsigned long long)tick);
    if (field && !write_file(stem + ".field.bin", field, field_bytes))
        return fail(MARL_ERR_INVALID_INPUT, "cannot write %s.field.bin: %s", stem.c_str(), std::strerror(errno));
    if (viewer_cells && !write_file(stem + ".cells.bin", viewer_cells, (size_t)n_cells * kViewerStride))
        return fail(MARL_ERR_INVALID_INPUT, "cannot write %s.cells.bin: %s", stem.c_str(), std::strerror(errno));
    return MARL_OK;
}

marl_status marl_ctx_write_ruleset_dumps(marl_ctx* c, const char* dir, uint64_t tick, int32_t mode) {
    if (!c || !dir) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (mode < MARL_RULESETS_LAYERS || mode > MARL_RULESETS_BOTH) return fail(MARL_ERR_INVALID_INPUT, "mode %d", mode);
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    const Grid g = c->g;
    const uint32_t n = c->n;
    cudaStream_t s = c->stream;
    std::vector<uint8_t> layers((size_t)g.Z * kLayerStride), canon;
    uint8_t* d_layers = nullptr;
    uint8_t* d_canon = nullptr;
    cudaError_t e = cudaSuccess;
    if (mode & MARL_RULESETS_LAYERS) {
        e = cudaMallocAsync((void**)&d_layers, layers.size(), s);
        if (e == cudaSuccess) {
            k_ruleset_layers<<<g.Z, kLayerThreads, 0, s>>>(c->t, n, d_layers);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(layers.data(), d_layers, layers.size(), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess && (mode & MARL_RULESETS_FULL) && n) {
        canon.resize((size_t)n * kCanonicalRecord);
        e = cudaMallocAsync((void**)&d_canon, canon.size(), s);
        if (e == cudaSuccess) {
            k_ruleset_canonical<<<(n + 127) / 128, 128, 0, s>>>(c->t, n, d_canon);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(canon.data(), d_canon, canon.size(), cudaMemcpyDeviceToHost, s);
    }
    if (d_layers) cudaFreeAsync(d_layers, s);
    if (d_canon) cudaFreeAsync(d_canon, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "marl_ctx_write_ruleset_dumps");
    c->d2h_bytes += layers.size() * ((mode & MARL_RULESETS_LAYERS) ? 1 : 0) + canon.size();
    return write_ruleset_files(dir, tick, g, mode, layers.data(), canon.data(), n);
}

marl_status marl_write_ruleset_dumps(const char* dir, uint64_t tick, int32_t gx, int32_t gy, int32_t gz,
                                     const marl_cell* cells, uint32_t n, int32_t mode) {
    if (!dir || (n && !cells)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (mode < MARL_RULESETS_LAYERS || mode > MARL_RULESETS_BOTH) return fail(MARL_ERR_INVALID_INPUT, "mode %d", mode);
    marl_status st = validate_dims(gx, gy, gz);
    if (st) return st;
    const Grid g{gx, gy, gz};
    for (uint32_t j = 0; j < n; ++j)
        if (cells[j].pos[2] >= gz) return fail(MARL_ERR_INVALID_INPUT, "cell %u: z %u outside the grid", j, cells[j].pos[2]);
    // Layer averages: f64 sums in cell order, then (sum / count) as f32 (binary_dump.rs:154-186).
    std::vector<uint8_t> layers((size_t)gz * kLayerStride, 0);
    std::vector<double> sums((size_t)gz * kLayerValues, 0.0);
    std::vector<uint32_t> counts(gz, 0);
    for (uint32_t j = 0; j < n; ++j) {
        const marl_ruleset& r = cells[j].ruleset;
        double* a = &sums[(size_t)cells[j].pos[2] * kLayerValues];
        int i = 0;
        for (const auto& x : r.receptors) a[i++] += x.k_half, a[i++] += x.n_hill, a[i++] += x.gain;
        for (const auto& x : r.transport) a[i++] += x.uptake_rate, a[i++] += x.secrete_rate;
        for (const auto& x : r.reactions) a[i++] += x.k_m, a[i++] += x.v_max, a[i++] += x.k_cat;
        for (const auto& x : r.effectors) a[i++] += x.threshold, a[i++] += x.rate;
        a[i++] += r.fate.division_energy, a[i++] += r.fate.death_energy, a[i++] += r.fate.quiescence_energy;
        a[i++] += r.fate.division_prep_ticks, a[i++] += r.hgt_propensity, a[i++] += r.mutation_rate;
        ++counts[cells[j].pos[2]];
    }
    for (int z = 0; z < gz; ++z) {
        uint8_t* rec = &layers[(size_t)z * kLayerStride];
        const uint16_t zz = (uint16_t)z;
        std::memcpy(rec, &zz, 2);
        std::memcpy(rec + 4, &counts[z], 4);
        for (int v = 0; v < kLayerValues; ++v) {
            const float avg = counts[z] ? (float)(sums[(size_t)z * kLayerValues + v] / (double)counts[z]) : 0.0f;
            std::memcpy(rec + 8 + 4 * v, &avg, 4);
        }
    }
    std::vector<uint8_t> canon;
    if (mode & MARL_RULESETS_FULL) {
        canon.assign((size_t)n * kCanonicalRecord, 0);
        for (uint32_t j = 0; j < n; ++j) {
            uint8_t* rec = &canon[(size_t)j * kCanonicalRecord];
            if ((st = marl_ruleset_pack_canonical(&cells[j].ruleset, rec))) return st;
            std::memcpy(rec + kCanonicalBytes, cells[j].pos, 6);
        }
    }
    return write_ruleset_files(dir, tick, g, mode, layers.data(), canon.data(), n);
}

}  // extern "C"
