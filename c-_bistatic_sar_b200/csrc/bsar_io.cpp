// bsar_io.cpp -- the files around the hot path.
//
//   matrix files   the reference's binary matrix format (src/binary_reader.cpp:8-99,
//                  src/data_export.cpp:71-138, 180-309): uint32 dimension count,
//                  uint32 complex flag, uint32 type-name length, char[16] type name,
//                  uint64 dimensions, then doubles (real / imaginary interleaved when
//                  complex).  2-D matrices are row-major; the 3-D image has x fastest.
//   scene files    a pulse matrix file staged through pinned memory straight into a
//                  resident scene; the simulator's [range row][pulse column] layout is
//                  transposed on the device (k_transpose_c128)
//   image files    the [x][y][z] device image permuted on the device to the file's
//                  x-fastest order, copied back once and written, with the grid axes as
//                  CSV files beside it like export3DComplexMatrix
//   ESRI ASCII     loadDEM's text grid parser (src/load_dem_simple.cpp:9-224), with its
//                  fallback DEM for .tif names and unreadable files
#include "runtime.hpp"

#include <cstdio>
#include <fstream>
#include <iomanip>
#include <sstream>

namespace {

constexpr uint32_t kMaxDims = 8;

struct FileCloser {
    FILE* f;
    ~FileCloser()
    {
        if (f) fclose(f);
    }
};

// Reads the header; leaves `f` at the first value.
void read_header(FILE* f, bsar_matrix_header* h)
{
    uint32_t nd = 0, cplx = 0, tlen = 0;
    char tname[16];
    if (fread(&nd, 4, 1, f) != 1) fail(BSAR_ERR_INVALID_ARG, "truncated file: no dimension count");
    if (fread(&cplx, 4, 1, f) != 1) fail(BSAR_ERR_INVALID_ARG, "truncated file: no complex flag");
    if (fread(&tlen, 4, 1, f) != 1) fail(BSAR_ERR_INVALID_ARG, "truncated file: no type-name length");
    if (fread(tname, 1, 16, f) != 16) fail(BSAR_ERR_INVALID_ARG, "truncated file: no type name");
    if (nd > kMaxDims) fail(BSAR_ERR_UNSUPPORTED, "%u dimensions (at most %u)", nd, kMaxDims);
    std::memset(h, 0, sizeof *h);
    h->ndims = nd;
    h->is_complex = cplx == 1 ? 1 : 0;           // the reader treats any other flag as real
    h->dtype_len = tlen < 16 ? tlen : 16;
    std::memcpy(h->dtype, tname, h->dtype_len);
    if (nd && fread(h->dims, 8, nd, f) != nd) fail(BSAR_ERR_INVALID_ARG, "truncated file: dimensions");
    uint64_t total = 1;
    for (uint32_t k = 0; k < nd; k++) {
        if (h->dims[k] && total > ((uint64_t)1 << 62) / h->dims[k]) fail(BSAR_ERR_INVALID_ARG, "dimensions overflow");
        total *= h->dims[k];
    }
    h->total = total;
}

FILE* open_read(const char* path)
{
    if (!path) fail(BSAR_ERR_INVALID_ARG, "path is NULL");
    FILE* f = fopen(path, "rb");
    if (!f) fail(BSAR_ERR_NOT_FOUND, "cannot open %s", path);
    return f;
}

void write_header(FILE* f, uint32_t nd, const uint64_t* dims, uint32_t cplx)
{
    const char name[] = "double";
    uint32_t tlen = 6;
    char tname[16] = {0};
    std::memcpy(tname, name, 6);
    bool ok = fwrite(&nd, 4, 1, f) == 1 && fwrite(&cplx, 4, 1, f) == 1 && fwrite(&tlen, 4, 1, f) == 1 &&
              fwrite(tname, 1, 16, f) == 16 && fwrite(dims, 8, nd, f) == nd;
    if (!ok) fail(BSAR_ERR_INVALID_ARG, "write failed");
}

// exportVector's text: fixed notation, 6 decimals, comma separated, one line.
void write_csv_vector(const std::string& path, const double* v, int64_t n)
{
    std::ofstream o(path);
    if (!o.is_open()) fail(BSAR_ERR_INVALID_ARG, "cannot create %s", path.c_str());
    o << std::fixed << std::setprecision(6);
    for (int64_t i = 0; i < n; i++) {
        if (i) o << ",";
        o << v[i];
    }
    o << std::endl;
}

// The image file plus, when axes are given, <path without extension>_grid_{x,y,z}.csv.
void write_image_file(const char* path, const double* xfast, int64_t nx, int64_t ny, int64_t nz, const double* gx,
                      const double* gy, const double* gz)
{
    FILE* f = fopen(path, "wb");
    if (!f) fail(BSAR_ERR_INVALID_ARG, "cannot create %s", path);
    FileCloser fc{f};
    const uint64_t dims[3] = {(uint64_t)nx, (uint64_t)ny, (uint64_t)nz};
    write_header(f, 3, dims, 1);
    const size_t n = 2 * (size_t)nx * ny * nz;
    if (fwrite(xfast, 8, n, f) != n) fail(BSAR_ERR_INVALID_ARG, "write failed");
    if (gx && gy && gz) {
        std::string p(path);
        const std::string base = p.substr(0, p.find_last_of('.'));
        write_csv_vector(base + "_grid_x.csv", gx, nx);
        write_csv_vector(base + "_grid_y.csv", gy, ny);
        write_csv_vector(base + "_grid_z.csv", gz, nz);
    }
}

struct PinnedBuf {
    void* p = nullptr;
    explicit PinnedBuf(size_t n)
    {
        cuda_check(cudaMallocHost(&p, n), "pinned buffer");
    }
    ~PinnedBuf()
    {
        if (p) cudaFreeHost(p);
    }
};

// Streams `bytes` of `f` into device memory `dst` through two pinned staging buffers, so
// reading the next chunk overlaps the copy of the previous one.
void file_to_device(bsar_ctx* ctx, FILE* f, char* dst, size_t bytes)
{
    constexpr size_t kChunk = size_t(16) << 20;
    PinnedBuf stage(2 * kChunk);
    cudaEvent_t ev[2];
    cuda_check(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming), "event");
    cuda_check(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming), "event");
    bool used[2] = {false, false};
    size_t done = 0;
    int k = 0;
    try {
        while (done < bytes) {
            const size_t n = std::min(kChunk, bytes - done);
            char* buf = static_cast<char*>(stage.p) + (size_t)k * kChunk;
            if (used[k]) cuda_check(cudaEventSynchronize(ev[k]), "staging wait");
            if (fread(buf, 1, n, f) != n) fail(BSAR_ERR_INVALID_ARG, "truncated file: values");
            cuda_check(cudaMemcpyAsync(dst + done, buf, n, cudaMemcpyHostToDevice, ctx->stream), "upload");
            cuda_check(cudaEventRecord(ev[k], ctx->stream), "event");
            used[k] = true;
            done += n;
            k ^= 1;
        }
        sync(ctx);
    } catch (...) {
        cudaStreamSynchronize(ctx->stream);
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        throw;
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
}

// ESRI ASCII grid as loadDEM parses it.  Returns the fallback flag.
int load_esri(const char* path, int64_t* nx_out, int64_t* ny_out, std::vector<double>& xv, std::vector<double>& yv,
              std::vector<double>& z)
{
    std::string name(path);
    std::ifstream file;
    const bool tif = name.find(".tif") != std::string::npos || name.find(".TIF") != std::string::npos;
    if (!tif) file.open(name);
    if (tif || !file.is_open()) {
        // the reference's stand-in terrain: 32 x 32 nodes over [-500, 500]^2, height 0
        const int M = 32;
        const double lim = 500.0, cell = (2.0 * lim) / (M - 1);
        xv.resize(M);
        yv.resize(M);
        for (int i = 0; i < M; i++) xv[i] = -lim + i * cell;
        for (int i = 0; i < M; i++) yv[i] = -lim + i * cell;
        z.assign((size_t)M * M, 0.0);
        *nx_out = M;
        *ny_out = M;
        return tif ? BSAR_DEM_FALLBACK_TIF : BSAR_DEM_FALLBACK_UNREADABLE;
    }
    int ncols = 0, nrows = 0, row = 0;
    double xll = 0.0, yll = 0.0, cell = 1.0, nodata = -9999.0;
    bool in_data = false;
    std::string line;
    auto parse_row = [&](const std::string& text) {
        std::istringstream vs(text);
        for (int col = 0; col < ncols; col++)
            if (!(vs >> z[(size_t)row * ncols + col])) z[(size_t)row * ncols + col] = nodata;
        row++;
    };
    while (std::getline(file, line)) {
        if (in_data) {
            if (row < nrows) parse_row(line);
            continue;
        }
        std::istringstream ts(line);
        std::string key;
        ts >> key;
        if (key == "ncols") ts >> ncols;
        else if (key == "nrows") ts >> nrows;
        else if (key == "xllcorner") ts >> xll;
        else if (key == "yllcorner") ts >> yll;
        else if (key == "cellsize") ts >> cell;
        else if (key == "NODATA_value" || key == "nodata_value") ts >> nodata;
        else {
            // first line that is not a header keyword: the grid starts here
            if (nrows < 0 || ncols < 0 || (nrows == 0 && ncols > 0))
                fail(BSAR_ERR_INVALID_ARG, "ESRI grid with %d rows and %d columns", nrows, ncols);
            in_data = true;
            z.assign((size_t)nrows * ncols, 0.0);
            xv.resize(ncols);
            yv.resize(nrows);
            for (int i = 0; i < ncols; i++) xv[i] = xll + i * cell;
            for (int i = 0; i < nrows; i++) yv[i] = yll + i * cell;
            if (nrows > 0) parse_row(line);
            else row++;
        }
    }
    *nx_out = ncols;
    *ny_out = nrows;
    int flags = 0;
    if (row != nrows) flags |= BSAR_DEM_ROWS_MISMATCH;
    return flags;
}

}  // namespace

extern "C" {

bsar_status bsar_matrix_read_header(const char* path, bsar_matrix_header* out)
{
    if (!out) return BSAR_ERR_INVALID_ARG;
    try {
        FileCloser fc{open_read(path)};
        read_header(fc.f, out);
        return BSAR_OK;
    } catch (const Error& e) {
        return e.status;
    }
}

bsar_status bsar_matrix_read(const char* path, double* out, uint64_t capacity)
{
    if (!out) return BSAR_ERR_INVALID_ARG;
    try {
        FileCloser fc{open_read(path)};
        bsar_matrix_header h;
        read_header(fc.f, &h);
        if (h.total > capacity) return BSAR_ERR_INVALID_ARG;
        if (h.is_complex) {
            if (fread(out, 16, h.total, fc.f) != h.total) return BSAR_ERR_INVALID_ARG;
        } else {
            // real values become complex with a zero imaginary part; expand in place from
            // the back
            if (fread(out, 8, h.total, fc.f) != h.total) return BSAR_ERR_INVALID_ARG;
            for (uint64_t i = h.total; i-- > 0;) {
                out[2 * i] = out[i];
                out[2 * i + 1] = 0.0;
            }
        }
        return BSAR_OK;
    } catch (const Error& e) {
        return e.status;
    }
}

bsar_status bsar_matrix_write(const char* path, uint32_t ndims, const uint64_t* dims, int32_t is_complex,
                              const double* data)
{
    if (!path || (ndims && !dims) || ndims > kMaxDims) return BSAR_ERR_INVALID_ARG;
    uint64_t total = 1;
    for (uint32_t k = 0; k < ndims; k++) total *= dims[k];
    if (total == 0 || !data) return BSAR_ERR_INVALID_ARG;     // exportComplexMatrix writes no empty matrix
    FILE* f = fopen(path, "wb");
    if (!f) return BSAR_ERR_INVALID_ARG;
    FileCloser fc{f};
    try {
        write_header(f, ndims, dims, is_complex ? 1u : 0u);
    } catch (const Error& e) {
        return e.status;
    }
    const uint64_t n = total * (is_complex ? 2 : 1);
    return fwrite(data, 8, n, f) == n ? BSAR_OK : BSAR_ERR_INVALID_ARG;
}

bsar_status bsar_scene_upload_file(bsar_ctx* ctx, const bsar_scene_desc* desc, const char* path, int32_t layout,
                                   bsar_scene_id* out)
{
    return guarded(ctx, [&] {
        if (!desc || !out) fail(BSAR_ERR_INVALID_ARG, "NULL argument");
        if (layout != BSAR_FILE_AS_IMAGER && layout != BSAR_FILE_ROW_MAJOR)
            fail(BSAR_ERR_INVALID_ARG, "unknown file layout %d", layout);
        FileCloser fc{open_read(path)};
        bsar_matrix_header h;
        read_header(fc.f, &h);
        if (h.ndims != 2) fail(BSAR_ERR_INVALID_ARG, "a pulse file holds a 2-D matrix (this one has %u dimensions)",
                               h.ndims);
        // the imager reads dims[0] as the fast-time length and dims[1] as the pulse count
        const int64_t ns = (int64_t)h.dims[0], np = (int64_t)h.dims[1];
        if (np != desc->n_pulses)
            fail(BSAR_ERR_INVALID_ARG, "the file holds %lld pulses, the trajectories %lld", (long long)np,
                 (long long)desc->n_pulses);
        bsar_scene_desc d = *desc;
        d.n_samples = ns;
        d.samples = nullptr;
        auto sc = make_scene(ctx, d, false);
        const size_t n = (size_t)np * ns;
        auto blob = dev_alloc(ctx, (h.is_complex ? 16 : 8) * n);
        file_to_device(ctx, fc.f, blob->as<char>(), (h.is_complex ? 16 : 8) * n);
        std::unique_ptr<DevBuf> cplx;
        const double2* src = blob->as<double2>();
        if (!h.is_complex) {
            cplx = dev_alloc(ctx, 16 * n);
            launched(ctx, launch_real_to_c128(blob->as<double>(), cplx->as<double2>(), (int64_t)n, ctx->stream),
                     "real to complex");
            src = cplx->as<double2>();
        }
        double2* dst = sc->samples->as<double2>();
        if (layout == BSAR_FILE_AS_IMAGER) {
            // the imager's reading (proc_test_script.cpp:326-331): element (range r, pulse p)
            // at p * ns + r, already pulse-major
            cuda_check(cudaMemcpyAsync(dst, src, 16 * n, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
        } else {
            // the file's own row-major [range][pulse] layout: element (r, p) at r * np + p
            launched(ctx, launch_transpose_c128(src, dst, ns, np, np, ns, 0, 0, 1, ctx->stream), "transpose");
        }
        sync(ctx);
        const uint64_t id = ctx->next_scene++;
        ctx->scenes[id] = std::move(sc);
        *out = id;
    });
}

bsar_status bsar_image_export(const char* path, const double* image, int64_t nx, int64_t ny, int64_t nz,
                              const double* gx, const double* gy, const double* gz)
{
    if (!path || !image || nx < 1 || ny < 1 || nz < 1) return BSAR_ERR_INVALID_ARG;
    try {
        std::vector<double> xf(2 * (size_t)nx * ny * nz);
        for (int64_t z = 0; z < nz; z++)
            for (int64_t y = 0; y < ny; y++)
                for (int64_t x = 0; x < nx; x++) {
                    const size_t s = 2 * (((size_t)x * ny + y) * nz + z), o = 2 * (((size_t)z * ny + y) * nx + x);
                    xf[o] = image[s];
                    xf[o + 1] = image[s + 1];
                }
        write_image_file(path, xf.data(), nx, ny, nz, gx, gy, gz);
        return BSAR_OK;
    } catch (const Error& e) {
        return e.status;
    } catch (const std::bad_alloc&) {
        return BSAR_ERR_OOM_BUDGET;
    }
}

bsar_status bsar_image_export_device(bsar_ctx* ctx, const char* path, const void* d_image, int64_t nx, int64_t ny,
                                     int64_t nz, const double* gx, const double* gy, const double* gz)
{
    return guarded(ctx, [&] {
        if (!path || !d_image || nx < 1 || ny < 1 || nz < 1) fail(BSAR_ERR_INVALID_ARG, "bad arguments");
        const size_t n = (size_t)nx * ny * nz;
        auto tmp = dev_alloc(ctx, 16 * n);
        // per y: the (x, z) plane, in[x][z] at x*ny*nz + y*nz + z -> out[z][x] at z*ny*nx + y*nx + x
        launched(ctx, launch_transpose_c128(static_cast<const double2*>(d_image), tmp->as<double2>(), nx, nz,
                                            ny * nz, ny * nx, nz, nx, ny, ctx->stream),
                 "image permute");
        PinnedBuf host(16 * n);
        cuda_check(cudaMemcpyAsync(host.p, tmp->p, 16 * n, cudaMemcpyDeviceToHost, ctx->stream), "download");
        sync(ctx);
        write_image_file(path, static_cast<const double*>(host.p), nx, ny, nz, gx, gy, gz);
    });
}

bsar_status bsar_dem_load_esri(const char* path, int64_t* nx, int64_t* ny, double* x_vec, double* y_vec, double* z,
                               int32_t* flags)
{
    if (!path || !nx || !ny) return BSAR_ERR_INVALID_ARG;
    try {
        std::vector<double> xv, yv, zz;
        int64_t cx = 0, cy = 0;
        const int f = load_esri(path, &cx, &cy, xv, yv, zz);
        if (flags) *flags = f;
        if (x_vec || y_vec || z) {
            if (!x_vec || !y_vec || !z || *nx < cx || *ny < cy) {
                *nx = cx;
                *ny = cy;
                return BSAR_ERR_INVALID_ARG;
            }
            std::memcpy(x_vec, xv.data(), 8 * xv.size());
            std::memcpy(y_vec, yv.data(), 8 * yv.size());
            std::memcpy(z, zz.data(), 8 * zz.size());
        }
        *nx = cx;
        *ny = cy;
        return BSAR_OK;
    } catch (const Error& e) {
        return e.status;
    } catch (const std::bad_alloc&) {
        return BSAR_ERR_OOM_BUDGET;
    }
}

}  // extern "C"
