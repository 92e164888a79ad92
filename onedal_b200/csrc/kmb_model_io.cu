// k-means model serialisation in oneDAL's binary archive format: the bytes
// that detail::serialize(kmeans::model<task::clustering>, binary_output_archive)
// writes (cpp/oneapi/dal/detail/archives.hpp:24-78, detail/serialization.hpp:
// 385-440), so a model saved by oneDAL loads here and a model saved here loads
// in oneDAL. The layout, field by field (all little-endian, no padding):
//
//   u32 magic 0x4441414F                              binary_output_archive::prologue
//   u8  1, u64 8010000000                             model impl (serialize_polymorphic,
//                                                     algo/kmeans/common.cpp:44-56, backend/serialization.hpp:194)
//   u8  1, u64 table id                               centroids table (table/common.cpp:239-241)
//     2020000000 (empty table): nothing follows       table/common.cpp:97-103
//     2030000000 (homogen table):                     table/backend/homogen_table_impl.hpp:136-138
//       u8 1, u64 2010000000                          simple metadata (table/common.cpp:133-146)
//       array<data_type>:    u64 1000000000, i32 0x0004 (int32), i64 4d, d x i32 (0x0100 f32 / 0x0200 f64)
//       array<feature_type>: u64 1000000000, i32 0x0004, i64 4d, d x i32 (3 = ratio)
//       array<byte_t>:       u64 1000000000, i32 0x0010 (uint8), i64 bytes, k*d values
//                                                     (detail/array_impl.cpp:26-37)
//       i64 row_count, i64 column_count, i32 layout (1 row-major, 2 column-major)
//
// Reading validates each id, element type and size the way oneDAL's
// deserialisation does; any mismatch or a read past the end is KMB_EINVAL (oneDAL:
// invalid_argument "Archive content does not match requested type").
#include "../../include/onedal_b200_kmeans.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr uint32_t kMagic = 0x4441414Fu;
constexpr uint64_t kArrayId = 1000000000ull;
constexpr uint64_t kSimpleMetaId = 2010000000ull;
constexpr uint64_t kEmptyTableId = 2020000000ull;
constexpr uint64_t kHomogenTableId = 2030000000ull;
constexpr uint64_t kKmeansModelId = 8010000000ull;
constexpr int32_t kDtInt32 = 0x0004, kDtUint8 = 0x0010, kDtF32 = 0x0100, kDtF64 = 0x0200;
constexpr int32_t kFeatureRatio = 3;
constexpr int32_t kRowMajor = 1, kColumnMajor = 2;

struct Writer {
    uint8_t *buf;
    int64_t cap;
    int64_t pos = 0;
    void put(const void *p, int64_t n) {
        if (buf && pos + n <= cap) std::memcpy(buf + pos, p, (size_t)n);
        pos += n;
    }
    template <typename T>
    void val(T v) {
        put(&v, sizeof(T));
    }
};

struct Reader {
    const uint8_t *buf;
    int64_t size;
    int64_t pos = 0;
    bool ok = true;
    void get(void *p, int64_t n) {
        if (!ok || n < 0 || n > size - pos) {
            ok = false;
            std::memset(p, 0, (size_t)(n > 0 ? n : 0));
            return;
        }
        std::memcpy(p, buf + pos, (size_t)n);
        pos += n;
    }
    template <typename T>
    T val() {
        T v{};
        get(&v, sizeof(T));
        return v;
    }
    // array header (detail/array_impl.cpp:39-53): id, element type, byte count
    bool array_header(int32_t expected_dtype, int64_t elem_size, int64_t *bytes) {
        if (val<uint64_t>() != kArrayId || !ok) return false;
        if (val<int32_t>() != expected_dtype || !ok) return false;
        *bytes = val<int64_t>();
        return ok && *bytes >= 0 && *bytes % elem_size == 0 && *bytes <= size - pos;
    }
};

int64_t elem_size(int dtype) { return dtype == KMB_F64 ? 8 : 4; }

// Writes the archive of a model with centroids C (host memory, k x d row-major;
// k == 0: a model without centroids). Returns the archive size.
int64_t write_model(uint8_t *buf, int64_t cap, int dtype, const void *C, int64_t k, int64_t d) {
    Writer w{buf, cap};
    w.val<uint32_t>(kMagic);
    w.val<uint8_t>(1);
    w.val<uint64_t>(kKmeansModelId);
    w.val<uint8_t>(1);
    if (k == 0) {
        w.val<uint64_t>(kEmptyTableId);
        return w.pos;
    }
    w.val<uint64_t>(kHomogenTableId);
    w.val<uint8_t>(1);
    w.val<uint64_t>(kSimpleMetaId);
    const int32_t dt = dtype == KMB_F64 ? kDtF64 : kDtF32;
    w.val<uint64_t>(kArrayId);
    w.val<int32_t>(kDtInt32);
    w.val<int64_t>(4 * d);
    for (int64_t j = 0; j < d; ++j) w.val<int32_t>(dt);
    w.val<uint64_t>(kArrayId);
    w.val<int32_t>(kDtInt32);
    w.val<int64_t>(4 * d);
    for (int64_t j = 0; j < d; ++j) w.val<int32_t>(kFeatureRatio);
    const int64_t bytes = k * d * elem_size(dtype);
    w.val<uint64_t>(kArrayId);
    w.val<int32_t>(kDtUint8);
    w.val<int64_t>(bytes);
    w.put(C, bytes);
    w.val<int64_t>(k);
    w.val<int64_t>(d);
    w.val<int32_t>(kRowMajor);
    return w.pos;
}

struct Parsed {
    int dtype = KMB_F32;
    int64_t k = 0, d = 0;
    int32_t layout = kRowMajor;
    const uint8_t *data = nullptr;  // inside the archive
};

bool parse_model(const uint8_t *buf, int64_t size, Parsed *out) {
    Reader r{buf, size};
    if (r.val<uint32_t>() != kMagic || !r.ok) return false;
    if (!r.val<uint8_t>() || r.val<uint64_t>() != kKmeansModelId || !r.ok) return false;
    if (!r.val<uint8_t>() || !r.ok) return false;
    const uint64_t table_id = r.val<uint64_t>();
    if (!r.ok) return false;
    if (table_id == kEmptyTableId) {
        out->k = out->d = 0;
        return true;
    }
    if (table_id != kHomogenTableId) return false;
    if (!r.val<uint8_t>() || r.val<uint64_t>() != kSimpleMetaId || !r.ok) return false;
    int64_t dt_bytes = 0, ft_bytes = 0, data_bytes = 0;
    if (!r.array_header(kDtInt32, 4, &dt_bytes)) return false;
    std::vector<int32_t> dtypes((size_t)(dt_bytes / 4));
    r.get(dtypes.data(), dt_bytes);
    if (!r.array_header(kDtInt32, 4, &ft_bytes)) return false;
    r.pos += ft_bytes;  // feature types do not change the centroids
    if (!r.array_header(kDtUint8, 1, &data_bytes)) return false;
    const uint8_t *data = buf + r.pos;
    r.pos += data_bytes;
    const int64_t rows = r.val<int64_t>(), cols = r.val<int64_t>();
    const int32_t layout = r.val<int32_t>();
    if (!r.ok || rows < 0 || cols < 0 || (int64_t)dtypes.size() != cols) return false;
    if (layout != kRowMajor && layout != kColumnMajor) return false;
    int dtype = KMB_F32;
    for (size_t j = 0; j < dtypes.size(); ++j) {
        if (dtypes[j] != kDtF32 && dtypes[j] != kDtF64) return false;
        if (dtypes[j] != dtypes[0]) return false;
        if (j == 0) dtype = dtypes[0] == kDtF64 ? KMB_F64 : KMB_F32;
    }
    if (rows > 0 && cols > 0 && data_bytes / elem_size(dtype) / cols != rows) return false;
    if (data_bytes != rows * cols * elem_size(dtype)) return false;
    out->dtype = dtype;
    out->k = rows;
    out->d = cols;
    out->layout = layout;
    out->data = data;
    return true;
}

// Row-major copy of the parsed centroids into host memory.
void copy_rows(const Parsed &p, void *dst) {
    const int64_t es = elem_size(p.dtype);
    if (p.layout == kRowMajor) {
        std::memcpy(dst, p.data, (size_t)(p.k * p.d * es));
        return;
    }
    uint8_t *o = (uint8_t *)dst;
    for (int64_t i = 0; i < p.k; ++i)
        for (int64_t j = 0; j < p.d; ++j) std::memcpy(o + (i * p.d + j) * es, p.data + (j * p.k + i) * es, (size_t)es);
}

}  // namespace

extern "C" {

int kmb_model_serialize(int dtype, int memory, const void *C, int64_t k, int64_t d, void *buf, int64_t capacity,
                        int64_t *size) {
    if (!size || (dtype != KMB_F32 && dtype != KMB_F64) || k < 0 || d < 0 || (k > 0 && (d == 0 || !C)))
        return KMB_EINVAL;
    if (memory != KMB_MEM_HOST && memory != KMB_MEM_DEVICE) return KMB_EINVAL;
    const int64_t need = write_model(nullptr, 0, dtype, nullptr, k, d);
    *size = need;
    if (!buf) return KMB_OK;  // size query
    if (capacity < need) return KMB_EINVAL;
    const void *host = C;
    std::vector<uint8_t> staging;
    if (memory == KMB_MEM_DEVICE && k > 0) {
        staging.resize((size_t)(k * d * elem_size(dtype)));
        if (cudaMemcpy(staging.data(), C, staging.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return KMB_ECUDA;
        host = staging.data();
    }
    write_model((uint8_t *)buf, capacity, dtype, host, k, d);
    return KMB_OK;
}

int kmb_model_deserialize(const void *buf, int64_t size, int *dtype, int64_t *k, int64_t *d, int memory, void *C_out,
                          int64_t capacity_bytes) {
    if (!buf || size < 0 || !dtype || !k || !d) return KMB_EINVAL;
    if (memory != KMB_MEM_HOST && memory != KMB_MEM_DEVICE) return KMB_EINVAL;
    Parsed p;
    if (!parse_model((const uint8_t *)buf, size, &p)) return KMB_EINVAL;
    *dtype = p.dtype;
    *k = p.k;
    *d = p.d;
    if (!C_out || p.k == 0) return KMB_OK;  // shape query, or a model without centroids
    const int64_t bytes = p.k * p.d * elem_size(p.dtype);
    if (capacity_bytes < bytes) return KMB_EINVAL;
    if (memory == KMB_MEM_HOST) {
        copy_rows(p, C_out);
        return KMB_OK;
    }
    if (p.layout == kRowMajor)
        return cudaMemcpy(C_out, p.data, (size_t)bytes, cudaMemcpyHostToDevice) == cudaSuccess ? KMB_OK : KMB_ECUDA;
    std::vector<uint8_t> rows((size_t)bytes);
    copy_rows(p, rows.data());
    return cudaMemcpy(C_out, rows.data(), (size_t)bytes, cudaMemcpyHostToDevice) == cudaSuccess ? KMB_OK : KMB_ECUDA;
}

int kmb_server_add_model_serialized(void *server, const void *buf, int64_t size, int32_t *model_id) {
    if (!server || !buf || !model_id) return KMB_EINVAL;
    Parsed p;
    if (!parse_model((const uint8_t *)buf, size, &p) || p.k == 0) return KMB_EINVAL;
    std::vector<float> C((size_t)(p.k * p.d));
    if (p.dtype == KMB_F32) {
        copy_rows(p, C.data());
    } else {  // the serving engine computes in float: double centroids are rounded once
        std::vector<double> c64((size_t)(p.k * p.d));
        copy_rows(p, c64.data());
        for (size_t i = 0; i < C.size(); ++i) C[i] = (float)c64[i];
    }
    return kmb_server_add_model(server, C.data(), p.k, p.d, model_id);
}

}  // extern "C"
