// output.cu -- dump files in the reference's formats (src/output.cpp): the
// ASCII `.dat` table (output_dat, src/output.cpp:65-224) and the binary
// appended-raw VTK StructuredGrid `.vts` (output_vts_binary,
// src/output.cpp:226-552), chosen by output_format like output()
// (src/output.cpp:555-572).
//
// The per-cell work -- velocities, gas pressure, v^2, B^2, the cell-centred
// divB diagnostic, cell-centre coordinates, and the reordering into the
// file's arrays -- runs on the GPU from q(0) in HBM, one slab of z planes at a
// time, into the context's staging buffer.  Each slab is copied to the host
// and written: the .vts blocks at their final file offsets (pwrite), the .dat
// lines formatted by host threads.  Only the file assembly is host code.
//
// how_output_async forms the whole domain's payload into its own HBM buffer
// on the main stream, copies it into pinned host memory on a side stream and
// writes the file from a host thread, so the steps queued after it overlap
// the copy and the write; how_output_wait joins the writer.
//
// The values are the reference's bit for bit: every operation is a separately
// rounded IEEE operation in the reference's evaluation order (the _rn
// intrinsics, which the compiler never fuses into FMAs), and the text uses
// the reference's stream format (std::scientific, precision 15 = "%.15e").
#include "how_internal.cuh"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <thread>
#include <vector>

namespace how {

namespace {

// bc_index_host (src/output.cpp:44-59): wrap over [lo, hi] when periodic,
// else clamp.
__device__ __forceinline__ int out_bc_index(int idx, int lo, int hi, int periodic) {
    if (periodic) {
        const int n = hi - lo + 1;
        int r = (idx - lo) % n;
        if (r < 0) r += n;
        return lo + r;
    }
    return idx < lo ? lo : (idx > hi ? hi : idx);
}

struct DumpArgs {
    Grid g;
    const double* q;          // q(0), device layout
    double* out;              // slab payload (staging buffer)
    int k0, nk;               // slab: padded planes k0 .. k0 + nk - 1
    int kofs;                 // global index of the first active plane (a part's kstart)
    int px, py, pz;           // periodic axes
    double dx, dy, dz, gam;
};

// The quantities of one active cell (src/output.cpp:110-187 and 284-354).
struct DumpCell {
    double x, y, z, rho, Mx, My, Mz, Bx, By, Bz, E, pg, vx, vy, vz, vv2, BB2, divB;
};

__device__ __forceinline__ DumpCell dump_cell(const DumpArgs& a, int i, int j, int k) {
    const Grid& g = a.g;
    const long long fs = g.fs, c = g.idx(i, j, k);
    DumpCell d;
    d.x = __dmul_rn(__dadd_rn((double)(i - 3), 0.5), a.dx);
    d.y = __dmul_rn(__dadd_rn((double)(j - 3), 0.5), a.dy);
    d.z = __dmul_rn(__dadd_rn((double)(a.kofs + k - 3), 0.5), a.dz);
    d.rho = a.q[c];
    d.Mx = a.q[fs + c]; d.My = a.q[2 * fs + c]; d.Mz = a.q[3 * fs + c];
    d.Bx = a.q[4 * fs + c]; d.By = a.q[5 * fs + c]; d.Bz = a.q[6 * fs + c];
    d.E = a.q[7 * fs + c];
    d.vx = __ddiv_rn(d.Mx, d.rho);
    d.vy = __ddiv_rn(d.My, d.rho);
    d.vz = __ddiv_rn(d.Mz, d.rho);
    d.vv2 = __dadd_rn(__dadd_rn(__dmul_rn(d.vx, d.vx), __dmul_rn(d.vy, d.vy)), __dmul_rn(d.vz, d.vz));
    d.BB2 = __dadd_rn(__dadd_rn(__dmul_rn(d.Bx, d.Bx), __dmul_rn(d.By, d.By)), __dmul_rn(d.Bz, d.Bz));
    // (gam - 1) * (E - 0.5 * rho * vv2 - 0.5 * BB2), left to right
    const double kin = __dmul_rn(__dmul_rn(0.5, d.rho), d.vv2);
    d.pg = __dmul_rn(__dsub_rn(a.gam, 1.0), __dsub_rn(__dsub_rn(d.E, kin), __dmul_rn(0.5, d.BB2)));
    // cell-centred central-difference divB: wrap when periodic, clamp when
    // open (one-sided differences over d at a clamped edge)
    double divB = 0.0;
    if (g.nx > 1) {
        const int im = out_bc_index(i - 1, 3, g.nx + 2, a.px), ip = out_bc_index(i + 1, 3, g.nx + 2, a.px);
        const double diff = __dsub_rn(a.q[4 * fs + g.idx(ip, j, k)], a.q[4 * fs + g.idx(im, j, k)]);
        divB = __dadd_rn(divB, __ddiv_rn(diff, (im == i || ip == i) ? a.dx : __dmul_rn(2.0, a.dx)));
    }
    if (g.ny > 1) {
        const int jm = out_bc_index(j - 1, 3, g.ny + 2, a.py), jp = out_bc_index(j + 1, 3, g.ny + 2, a.py);
        const double diff = __dsub_rn(a.q[5 * fs + g.idx(i, jp, k)], a.q[5 * fs + g.idx(i, jm, k)]);
        divB = __dadd_rn(divB, __ddiv_rn(diff, (jm == j || jp == j) ? a.dy : __dmul_rn(2.0, a.dy)));
    }
    if (g.nz > 1) {
        const int km = out_bc_index(k - 1, 3, g.nz + 2, a.pz), kp = out_bc_index(k + 1, 3, g.nz + 2, a.pz);
        const double diff = __dsub_rn(a.q[6 * fs + g.idx(i, j, kp)], a.q[6 * fs + g.idx(i, j, km)]);
        divB = __dadd_rn(divB, __ddiv_rn(diff, (km == k || kp == k) ? a.dz : __dmul_rn(2.0, a.dz)));
    }
    d.divB = divB;
    return d;
}

// .vts slab: the ten appended arrays of src/output.cpp:380-395 in file order,
// each holding this slab's points (x fastest): rho, pressure, energy, v2, B2,
// divB (1 component), velocity, magnetic_field, momentum, points (3).
constexpr int kVtsComps = 18;
__global__ void k_dump_vts(DumpArgs a) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i > a.g.nx + 2) return;
    const int j = 3 + blockIdx.y, k = a.k0 + blockIdx.z;
    const DumpCell d = dump_cell(a, i, j, k);
    const long long n = (long long)a.g.nx * a.g.ny * a.nk;
    const long long p = (i - 3) + (long long)a.g.nx * ((j - 3) + (long long)a.g.ny * (k - a.k0));
    double* o = a.out;
    o[p] = d.rho;
    o[n + p] = d.pg;
    o[2 * n + p] = d.E;
    o[3 * n + p] = d.vv2;
    o[4 * n + p] = d.BB2;
    o[5 * n + p] = d.divB;
    double* v = o + 6 * n + 3 * p;
    v[0] = d.vx; v[1] = d.vy; v[2] = d.vz;
    v += 3 * n;
    v[0] = d.Bx; v[1] = d.By; v[2] = d.Bz;
    v += 3 * n;
    v[0] = d.Mx; v[1] = d.My; v[2] = d.Mz;
    v += 3 * n;
    v[0] = d.x; v[1] = d.y; v[2] = d.z;
}

// .dat slab: the 16 floating-point columns of a row (src/output.cpp:190-211)
// per cell, cells in file order.
constexpr int kDatCols = 16;
__global__ void k_dump_dat(DumpArgs a) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i > a.g.nx + 2) return;
    const int j = 3 + blockIdx.y, k = a.k0 + blockIdx.z;
    const DumpCell d = dump_cell(a, i, j, k);
    const long long p = (i - 3) + (long long)a.g.nx * ((j - 3) + (long long)a.g.ny * (k - a.k0));
    double* o = a.out + kDatCols * p;
    o[0] = d.x; o[1] = d.y; o[2] = d.z;
    o[3] = d.rho; o[4] = d.Mx; o[5] = d.My; o[6] = d.Mz;
    o[7] = d.Bx; o[8] = d.By; o[9] = d.Bz; o[10] = d.E;
    o[11] = d.pg; o[12] = d.vx; o[13] = d.vy; o[14] = d.vz; o[15] = d.divB;
}

// The stream's std::scientific, precision 15 rendering of a double.
inline void put_sci(std::string& s, double v) {
    char b[40];
    const int n = std::snprintf(b, sizeof(b), "%.15e", v);
    s.append(b, (size_t)n);
}

inline void put_int(std::string& s, long long v) {
    char b[24];
    const int n = std::snprintf(b, sizeof(b), "%lld", v);
    s.append(b, (size_t)n);
}

// Full write of n bytes at offset off; false on an I/O error.
bool pwrite_all(int fd, const void* data, size_t n, off_t off) {
    const char* p = static_cast<const char*>(data);
    while (n > 0) {
        const ssize_t w = ::pwrite(fd, p, n, off);
        if (w < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        p += w; n -= (size_t)w; off += w;
    }
    return true;
}

// make_output_filename (src/output.cpp:21-38): <dir>/dumpNNNNNN<ext>, or for
// one part of a decomposed domain, the MPI form <dir>/dumpNNNNNN_rankRRRRRR<ext>
std::string dump_file(int step, const char* ext, int rank) {
    char b[48];
    if (rank >= 0) std::snprintf(b, sizeof(b), "dump%06d_rank%06d%s", step, rank, ext);
    else std::snprintf(b, sizeof(b), "dump%06d%s", step, ext);
    return b;
}

std::string dump_name(const char* dir, int step, const char* ext, int rank) {
    const std::string b = dump_file(step, ext, rank);
    std::string d = dir ? dir : "output";
    return d.empty() ? b : d + "/" + b;
}

int make_dirs(const std::string& dir) {
    if (dir.empty()) return HOW_OK;
    std::string cur;
    for (size_t i = 0; i <= dir.size(); ++i) {
        if (i == dir.size() || dir[i] == '/') {
            if (!cur.empty() && ::mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST) {
                set_error("cannot create directory %s: %s", cur.c_str(), std::strerror(errno));
                return HOW_ERR_ARG;
            }
        }
        if (i < dir.size()) cur.push_back(dir[i]);
    }
    return HOW_OK;
}

// Planes per slab: the payload fits the staging buffer (8 fields, always room
// for one plane's 18 values per cell) and, unless a single plane is larger,
// at most 2^26 doubles (512 MB) are held on the host at once.
int slab_planes(const Ctx& c, int per_cell) {
    const Grid& g = c.g;
    const long long cap = std::min<long long>(8LL * g.fs, 1LL << 26);
    long long k = cap / ((long long)per_cell * g.nx * g.ny);
    if (k < 1) k = 1;
    if (k > g.nz) k = g.nz;
    return (int)k;
}

DumpArgs dump_args(const Ctx& c) {
    DumpArgs a;
    a.g = c.g;
    a.q = c.q[0];
    a.out = c.stage_buf;
    a.k0 = 3; a.nk = 0;
    a.kofs = c.part >= 0 ? c.kstart : 0;
    a.px = c.p.bc[0] == HOW_BC_PERIODIC;
    a.py = c.p.bc[1] == HOW_BC_PERIODIC;
    a.pz = c.p.bc[2] == HOW_BC_PERIODIC;
    a.dx = c.p.dx; a.dy = c.p.dy; a.dz = c.p.dz; a.gam = c.p.gam;
    return a;
}

// Where a file's cells sit in the whole domain: the header fields the
// reference fills from its MPI decomposition (cart_rank, gnx/gny/gnz,
// istart/jstart/kstart, src/parameters.hpp:20, 59, 71).  A single domain is
// rank 0 at the origin; a part of a z-decomposed group is rank `part` (the
// Cartesian rank of a 1 x 1 x P layout) starting at global plane kstart.
struct PieceInfo {
    int rank, gnx, gny, gnz, istart, jstart, kstart;
};

PieceInfo piece_of(const Ctx& c) {
    PieceInfo pi{0, c.g.nx, c.g.ny, c.g.nz, 0, 0, 0};
    if (c.part >= 0) { pi.rank = c.part; pi.gnz = c.gnz; pi.kstart = c.kstart; }
    return pi;
}

// Supplies the payload of active planes [k0, k0 + nk) in the kernels' slab
// layout, host-resident.
using SlabFn = std::function<int(int k0, int nk, const double** data)>;

int assemble_vts(const Grid& g, const PieceInfo& pi, int step, double time, const std::string& path, int K,
                 const SlabFn& slab) {
    const long long npts = (long long)g.nx * g.ny * g.nz;
    // appended blocks: [u64 bytes][payload], offsets from the byte after "_"
    const int ncomp[10] = {1, 1, 1, 1, 1, 1, 3, 3, 3, 3};
    unsigned long long off[10], pos = 0;
    for (int b = 0; b < 10; ++b) { off[b] = pos; pos += 8 + 8ULL * ncomp[b] * npts; }
    const unsigned long long payload = pos;

    std::string h;
    h += "<?xml version=\"1.0\"?>\n";
    h += "<VTKFile type=\"StructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    h += "  <StructuredGrid WholeExtent=\"0 "; put_int(h, pi.gnx - 1); h += " 0 "; put_int(h, pi.gny - 1);
    h += " 0 "; put_int(h, pi.gnz - 1); h += "\">\n";
    h += "    <Piece Extent=\""; put_int(h, pi.istart); h += " "; put_int(h, pi.istart + g.nx - 1);
    h += " "; put_int(h, pi.jstart); h += " "; put_int(h, pi.jstart + g.ny - 1);
    h += " "; put_int(h, pi.kstart); h += " "; put_int(h, pi.kstart + g.nz - 1); h += "\">\n";
    h += "      <FieldData>\n";
    h += "        <DataArray type=\"Float64\" Name=\"time\" NumberOfTuples=\"1\" format=\"ascii\">\n";
    h += "          "; put_sci(h, time); h += "\n";
    h += "        </DataArray>\n";
    h += "        <DataArray type=\"Int32\" Name=\"step\" NumberOfTuples=\"1\" format=\"ascii\">\n";
    h += "          "; put_int(h, step); h += "\n";
    h += "        </DataArray>\n";
    h += "        <DataArray type=\"Int32\" Name=\"rank\" NumberOfTuples=\"1\" format=\"ascii\">\n";
    h += "          "; put_int(h, pi.rank); h += "\n";
    h += "        </DataArray>\n";
    h += "        <DataArray type=\"Int32\" Name=\"global_start_index\" NumberOfComponents=\"3\" "
         "NumberOfTuples=\"1\" format=\"ascii\">\n";
    h += "          "; put_int(h, pi.istart); h += " "; put_int(h, pi.jstart); h += " "; put_int(h, pi.kstart);
    h += "\n";
    h += "        </DataArray>\n";
    h += "      </FieldData>\n";
    h += "      <PointData>\n";
    const char* names[9] = {"rho", "pressure", "energy", "v2", "B2", "divB", "velocity", "magnetic_field",
                            "momentum"};
    for (int b = 0; b < 9; ++b) {
        h += "        <DataArray type=\"Float64\" Name=\""; h += names[b];
        h += "\" NumberOfComponents=\""; put_int(h, ncomp[b]);
        h += "\" format=\"appended\" offset=\""; put_int(h, (long long)off[b]); h += "\"/>\n";
    }
    h += "      </PointData>\n";
    h += "      <CellData>\n";
    h += "      </CellData>\n";
    h += "      <Points>\n";
    h += "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"appended\" offset=\"";
    put_int(h, (long long)off[9]); h += "\"/>\n";
    h += "      </Points>\n";
    h += "    </Piece>\n";
    h += "  </StructuredGrid>\n";
    h += "  <AppendedData encoding=\"raw\">\n";
    h += "_";
    const off_t base = (off_t)h.size();
    const char* tail = "\n  </AppendedData>\n</VTKFile>\n";

    const int fd = ::open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0666);
    if (fd < 0) { set_error("cannot open output file %s: %s", path.c_str(), std::strerror(errno)); return HOW_ERR_ARG; }
    bool ok = pwrite_all(fd, h.data(), h.size(), 0);
    for (int b = 0; b < 10 && ok; ++b) {
        const unsigned long long nbytes = 8ULL * ncomp[b] * npts;
        ok = pwrite_all(fd, &nbytes, 8, base + (off_t)off[b]);
    }
    ok = ok && pwrite_all(fd, tail, std::strlen(tail), base + (off_t)payload);
    int rc = HOW_OK;
    for (int k0 = 0; k0 < g.nz && ok && rc == HOW_OK; k0 += K) {
        const int nk = std::min(K, g.nz - k0);
        const long long n = (long long)g.nx * g.ny * nk;
        const double* src = nullptr;
        rc = slab(k0, nk, &src);
        if (rc) break;
        const long long first = (long long)g.nx * g.ny * k0;   // this slab's first point
        for (int b = 0; b < 10 && ok; ++b) {
            const off_t at = base + (off_t)off[b] + 8 + (off_t)(8LL * ncomp[b] * first);
            ok = pwrite_all(fd, src, (size_t)(8LL * ncomp[b] * n), at);
            src += ncomp[b] * n;
        }
    }
    if (::close(fd) != 0) ok = false;
    if (rc) return rc;
    if (!ok) { set_error("write to %s failed: %s", path.c_str(), std::strerror(errno)); return HOW_ERR_ARG; }
    return HOW_OK;
}

int assemble_dat(const Grid& g, const PieceInfo& pi, int step, double time, const std::string& path, int K,
                 const SlabFn& slab) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { set_error("cannot open output file %s: %s", path.c_str(), std::strerror(errno)); return HOW_ERR_ARG; }
    std::string h;
    h += "# step = "; put_int(h, step); h += "\n";
    h += "# time = "; put_sci(h, time); h += "\n";
    h += "# rank = "; put_int(h, pi.rank); h += "\n";
    h += "# local_active_size = "; put_int(h, g.nx); h += " "; put_int(h, g.ny); h += " "; put_int(h, g.nz); h += "\n";
    h += "# global_active_size = "; put_int(h, pi.gnx); h += " "; put_int(h, pi.gny); h += " "; put_int(h, pi.gnz);
    h += "\n";
    h += "# global_start_index = "; put_int(h, pi.istart); h += " "; put_int(h, pi.jstart); h += " ";
    put_int(h, pi.kstart); h += "\n";
    h += "# columns: ig jg kg il jl kl x y z rho Mx My Mz Bx By Bz E pg vx vy vz divB\n";
    bool ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
    int rc = HOW_OK;
    for (int k0 = 0; k0 < g.nz && ok && rc == HOW_OK; k0 += K) {
        const int nk = std::min(K, g.nz - k0);
        const double* src = nullptr;
        rc = slab(k0, nk, &src);
        if (rc) break;
        // one text row per (j, k) line of the slab, formatted in parallel
        const int rows = g.ny * nk;
        std::vector<std::string> text((size_t)rows);
#pragma omp parallel for schedule(dynamic, 4)
        for (int r = 0; r < rows; ++r) {
            const int jl = r % g.ny, kl = k0 + r / g.ny;
            std::string& s = text[(size_t)r];
            s.reserve((size_t)g.nx * 400);
            for (int il = 0; il < g.nx; ++il) {
                const double* v = src + kDatCols * ((long long)r * g.nx + il);
                put_int(s, pi.istart + il); s += ' '; put_int(s, pi.jstart + jl); s += ' ';
                put_int(s, pi.kstart + kl); s += ' ';
                put_int(s, il); s += ' '; put_int(s, jl); s += ' '; put_int(s, kl);
                for (int m = 0; m < kDatCols; ++m) { s += ' '; put_sci(s, v[m]); }
                s += '\n';
            }
        }
        for (int r = 0; r < rows && ok; ++r) ok = std::fwrite(text[r].data(), 1, text[r].size(), f) == text[r].size();
    }
    if (std::fclose(f) != 0) ok = false;
    if (rc) return rc;
    if (!ok) { set_error("write to %s failed", path.c_str()); return HOW_ERR_ARG; }
    return HOW_OK;
}

void launch_dump(Ctx& c, DumpArgs a, bool dat) {
    const dim3 grid((c.g.nx + 127) / 128, c.g.ny, a.nk);
    if (dat) k_dump_dat<<<grid, 128, 0, c.stream>>>(a);
    else k_dump_vts<<<grid, 128, 0, c.stream>>>(a);
    ++c.launches;
}

// Checks the context and the format; *skip when output_format is "none".
int dump_prologue(how_ctx* c, const char* dir, bool* dat, bool* skip, std::string* path, int step) {
    if (!c) { set_error("null context"); return HOW_ERR_ARG; }
    HOW_CUDA_CHECK(cudaSetDevice(c->dev));
    const std::string fmt = c->p.output_format;
    *skip = fmt == "none";
    if (*skip) return HOW_OK;
    *dat = fmt == "dat";
    if (!*dat && fmt != "vtk" && fmt != "vts") {
        // the reference prints the options and aborts (src/output.cpp:566-570)
        set_error("unknown output_format = %s (available options: dat, vtk, none)", fmt.c_str());
        return HOW_ERR_ARG;
    }
    const int rc = make_dirs(dir ? dir : "output");
    if (rc) return rc;
    *path = dump_name(dir, step, *dat ? ".dat" : ".vts", c->part);
    return HOW_OK;
}

}  // namespace

// Asynchronous dumps: the payload of the whole domain in HBM, copied on a side
// stream into pinned host memory once the main stream has formed it, and
// written by a host thread.  One dump is in flight per context.
struct DumpJob {
    double* dev = nullptr;
    size_t dev_n = 0;
    double* host = nullptr;
    size_t host_n = 0;
    cudaStream_t side = nullptr;
    cudaEvent_t formed = nullptr, copied = nullptr;
    std::thread writer;
    bool busy = false;
    int rc = HOW_OK;
    std::string err;
};

int dump_join(Ctx& c) {
    DumpJob* j = c.dump;
    if (!j || !j->busy) return HOW_OK;
    j->writer.join();
    j->busy = false;
    if (j->rc) set_error("%s", j->err.c_str());
    return j->rc;
}

void dump_release(Ctx& c) {
    if (!c.dump) return;
    dump_join(c);
    DumpJob* j = c.dump;
    if (j->dev) cudaFree(j->dev);
    if (j->host) cudaFreeHost(j->host);
    if (j->formed) cudaEventDestroy(j->formed);
    if (j->copied) cudaEventDestroy(j->copied);
    if (j->side) cudaStreamDestroy(j->side);
    delete j;
    c.dump = nullptr;
}

// The master file of a decomposed domain's .vts pieces: a VTK XML
// PStructuredGrid over the whole extent, declaring the pieces' arrays and
// listing each piece's extent and file (relative to the master's directory).
// The reference lists this file as a to-do (README.md:758): its MPI ranks
// write only their pieces.  As there, a piece's points are its own cell
// centres, so neighbouring pieces do not share a layer of points.
int write_pvts(const how_params& gp, int nparts, const int* kstart, const int* nzl, int step, const char* dir) {
    std::string h;
    h += "<?xml version=\"1.0\"?>\n";
    h += "<VTKFile type=\"PStructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    h += "  <PStructuredGrid WholeExtent=\"0 "; put_int(h, gp.nx - 1); h += " 0 "; put_int(h, gp.ny - 1);
    h += " 0 "; put_int(h, gp.nz - 1); h += "\" GhostLevel=\"0\">\n";
    h += "    <PPointData>\n";
    const char* names[9] = {"rho", "pressure", "energy", "v2", "B2", "divB", "velocity", "magnetic_field",
                            "momentum"};
    for (int b = 0; b < 9; ++b) {
        h += "      <PDataArray type=\"Float64\" Name=\""; h += names[b];
        h += "\" NumberOfComponents=\""; put_int(h, b < 6 ? 1 : 3); h += "\"/>\n";
    }
    h += "    </PPointData>\n";
    h += "    <PCellData>\n";
    h += "    </PCellData>\n";
    h += "    <PPoints>\n";
    h += "      <PDataArray type=\"Float64\" NumberOfComponents=\"3\"/>\n";
    h += "    </PPoints>\n";
    for (int p = 0; p < nparts; ++p) {
        h += "    <Piece Extent=\"0 "; put_int(h, gp.nx - 1); h += " 0 "; put_int(h, gp.ny - 1);
        h += " "; put_int(h, kstart[p]); h += " "; put_int(h, kstart[p] + nzl[p] - 1);
        h += "\" Source=\""; h += dump_file(step, ".vts", p); h += "\"/>\n";
    }
    h += "  </PStructuredGrid>\n";
    h += "</VTKFile>\n";
    const std::string path = dump_name(dir, step, ".pvts", -1);
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { set_error("cannot open output file %s: %s", path.c_str(), std::strerror(errno)); return HOW_ERR_ARG; }
    const bool ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
    if (std::fclose(f) != 0 || !ok) { set_error("write to %s failed", path.c_str()); return HOW_ERR_ARG; }
    return HOW_OK;
}

}  // namespace how

using namespace how;

extern "C" int how_output(how_ctx* c, int step, double time, const char* dir) {
    bool dat = false, skip = false;
    std::string path;
    int rc = dump_prologue(c, dir, &dat, &skip, &path, step);
    if (rc || skip) return rc;
    HOW_CUDA_CHECK(cudaStreamSynchronize(c->stream));   // q(0) final
    DumpArgs a = dump_args(*c);
    const int K = slab_planes(*c, dat ? kDatCols : kVtsComps);
    std::vector<double> host;
    Ctx& cx = *c;
    SlabFn slab = [&](int k0, int nk, const double** data) -> int {
        a.k0 = 3 + k0;
        a.nk = nk;
        launch_dump(cx, a, dat);
        const size_t n = (size_t)(dat ? kDatCols : kVtsComps) * cx.g.nx * cx.g.ny * nk;
        host.resize(n);
        HOW_CUDA_CHECK(cudaGetLastError());
        HOW_CUDA_CHECK(cudaMemcpyAsync(host.data(), cx.stage_buf, n * sizeof(double), cudaMemcpyDeviceToHost,
                                       cx.stream));
        HOW_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
        *data = host.data();
        return HOW_OK;
    };
    const PieceInfo pi = piece_of(*c);
    return dat ? assemble_dat(c->g, pi, step, time, path, K, slab)
               : assemble_vts(c->g, pi, step, time, path, K, slab);
}

extern "C" int how_output_async(how_ctx* c, int step, double time, const char* dir) {
    bool dat = false, skip = false;
    std::string path;
    int rc = dump_prologue(c, dir, &dat, &skip, &path, step);
    if (rc || skip) return rc;
    if ((rc = dump_join(*c))) return rc;   // the previous dump first
    if (!c->dump) c->dump = new DumpJob();
    DumpJob* j = c->dump;
    const Grid& g = c->g;
    const size_t n = (size_t)(dat ? kDatCols : kVtsComps) * g.nx * g.ny * g.nz;
    if (j->dev_n < n) {
        if (j->dev) cudaFree(j->dev);
        j->dev = nullptr; j->dev_n = 0;
        HOW_CUDA_CHECK(cudaMalloc(&j->dev, n * sizeof(double)));
        j->dev_n = n;
    }
    if (j->host_n < n) {
        if (j->host) cudaFreeHost(j->host);
        j->host = nullptr; j->host_n = 0;
        HOW_CUDA_CHECK(cudaMallocHost(&j->host, n * sizeof(double)));
        j->host_n = n;
    }
    if (!j->side) HOW_CUDA_CHECK(cudaStreamCreateWithFlags(&j->side, cudaStreamNonBlocking));
    if (!j->formed) HOW_CUDA_CHECK(cudaEventCreateWithFlags(&j->formed, cudaEventDisableTiming));
    if (!j->copied) HOW_CUDA_CHECK(cudaEventCreateWithFlags(&j->copied, cudaEventDisableTiming));
    // the whole domain as one slab, ordered after the steps already queued
    DumpArgs a = dump_args(*c);
    a.out = j->dev;
    a.k0 = 3;
    a.nk = g.nz;
    launch_dump(*c, a, dat);
    HOW_CUDA_CHECK(cudaGetLastError());
    HOW_CUDA_CHECK(cudaEventRecord(j->formed, c->stream));
    HOW_CUDA_CHECK(cudaStreamWaitEvent(j->side, j->formed, 0));
    HOW_CUDA_CHECK(cudaMemcpyAsync(j->host, j->dev, n * sizeof(double), cudaMemcpyDeviceToHost, j->side));
    HOW_CUDA_CHECK(cudaEventRecord(j->copied, j->side));
    j->rc = HOW_OK;
    j->err.clear();
    const int dev = c->dev;
    const Grid gg = g;
    const PieceInfo pi = piece_of(*c);
    j->writer = std::thread([j, dev, gg, pi, step, time, path, dat]() {
        int r = HOW_OK;
        cudaError_t e = cudaSetDevice(dev);
        if (e == cudaSuccess) e = cudaEventSynchronize(j->copied);
        if (e != cudaSuccess) {
            r = cuda_fail(e, "dump copy");
        } else {
            const double* host = j->host;
            SlabFn whole = [host](int, int, const double** data) -> int { *data = host; return HOW_OK; };
            r = dat ? assemble_dat(gg, pi, step, time, path, gg.nz, whole)
                    : assemble_vts(gg, pi, step, time, path, gg.nz, whole);
        }
        j->rc = r;
        if (r) j->err = how_last_error();
    });
    j->busy = true;
    return HOW_OK;
}

extern "C" int how_output_wait(how_ctx* c) {
    if (!c) { set_error("null context"); return HOW_ERR_ARG; }
    return dump_join(*c);
}
