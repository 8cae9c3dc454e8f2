// Binary snapshot output from device state: the reference's field and cell
// dumps (crates/marl-output/src/binary_dump.rs:109-120) and run_meta.json
// (crates/marl-format/src/lib.rs:130-218), uncompressed.
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
    const std::string meta_path = base + "/run_meta.json";
    char meta[1024];
    std::snprintf(meta, sizeof(meta),
                  "{\n  \"grid_x\": %d,\n  \"grid_y\": %d,\n  \"grid_z\": %d,\n  \"s_ext\": %d,\n  \"m_int\": %d,\n"
                  "  \"field_dtype\": \"f32\",\n  \"field_layout\": \"z_y_x_species\",\n"
                  "  \"field_byte_len\": %llu,\n  \"cell_record_stride\": %u,\n  \"endianness\": \"little\",\n"
                  "  \"binary_format_version\": 2,\n  \"binary_compression\": \"none\",\n"
                  "  \"binary_compression_level\": 0,\n  \"write_binary_field\": %s,\n  \"write_binary_cells\": %s,\n"
                  "  \"field_file_pattern\": \"tick_<T>.field.bin\",\n  \"cell_file_pattern\": \"tick_<T>.cells.bin\"\n}\n",
                  gx, gy, gz, MARL_S_EXT, MARL_M_INT, (unsigned long long)field_bytes, kViewerStride,
                  field ? "true" : "false", viewer_cells ? "true" : "false");
    if (!write_file(meta_path, meta, std::strlen(meta)))
        return fail(MARL_ERR_INVALID_INPUT, "cannot write %s: %s", meta_path.c_str(), std::strerror(errno));
    const std::string stem = base + "/tick_" + std::to_string((unsigned long long)tick);
    if (field && !write_file(stem + ".field.bin", field, field_bytes))
        return fail(MARL_ERR_INVALID_INPUT, "cannot write %s.field.bin: %s", stem.c_str(), std::strerror(errno));
    if (viewer_cells && !write_file(stem + ".cells.bin", viewer_cells, (size_t)n_cells * kViewerStride))
        return fail(MARL_ERR_INVALID_INPUT, "cannot write %s.cells.bin: %s", stem.c_str(), std::strerror(errno));
    return MARL_OK;
}

}  // extern "C"
