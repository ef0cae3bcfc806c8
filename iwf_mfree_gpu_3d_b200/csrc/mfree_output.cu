// mfree_output.cu -- output in the reference's file formats.
//
// Reference writers replaced:
//   vtk_writer_write(particle_gpu*)       vtk_writer.cpp:78-262  particles (legacy VTK, ASCII)
//   vtk_writer_write_unified(tools, ...)  vtk_writer.cpp:307-386 tool meshes, one file
//   vtk_writer_write_blanking()           vtk_writer.cpp:22-77   blanking box
//   tool_forces::report                   tool_3d_gpu.cu:53-69   force log line
//
// The reference copies every field back with blocking cudaMemcpy calls and
// formats the file before the next step starts.  Here the particle output
// takes a snapshot of the state with device-to-device copies on the step
// stream (a few tens of microseconds for a million particles), copies the
// snapshot to pinned host memory on a stream of its own, and formats and
// writes the file on a host thread: the caller keeps stepping meanwhile.  One
// particle output per context is in flight; the next call (or
// mfree_output_wait, or mfree_destroy) waits for it.  The text is the
// reference's: the same header, sections, order and printf conversions.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "mfree_ctx.h"

using namespace mfree;
using namespace mfree::host;

// snapshot arrays (float4 each, n_init entries)
enum { SN_POS = 0, SN_VEL, SN_SA, SN_SB, SN_DSB, SN_FC, SN_FT, SN_RV, SN_N };

struct OutputJob {
    int device = 0;
    int n = 0;
    cudaStream_t stream = nullptr;  // the copy to the host, off the step stream
    cudaEvent_t snap = nullptr;     // the snapshot is taken
    float4 *d_snap = nullptr;
    float4 *h_snap = nullptr;       // pinned
    float c0sq = 0.f, rho0 = 0.f;
    std::string path;
    std::thread worker;
    int status = MFREE_OK;
    std::string err;
};

namespace {

// printf into a growing buffer
struct Text {
    std::vector<char> b;
    void add(const char *fmt, ...) __attribute__((format(printf, 2, 3)));
};
void Text::add(const char *fmt, ...) {
    char tmp[256];
    va_list ap;
    va_start(ap, fmt);
    const int k = vsnprintf(tmp, sizeof(tmp), fmt, ap);
    va_end(ap);
    if (k > 0) b.insert(b.end(), tmp, tmp + std::min<int>(k, int(sizeof(tmp)) - 1));
}

// the body of one section for particles [lo, hi), formatted in parallel
// chunks and concatenated in order
template <class F> void sections(FILE *fp, int n, F &&line) {
    const int nt = std::max(1, std::min<int>(8, int(std::thread::hardware_concurrency())));
    const int chunk = (n + nt - 1) / nt;
    std::vector<Text> parts(nt);
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
        th.emplace_back([&, t] {
            const int lo = t * chunk, hi = std::min(n, lo + chunk);
            for (int i = lo; i < hi; i++) line(parts[t], i);
        });
    for (auto &x : th) x.join();
    for (auto &p : parts) fwrite(p.b.data(), 1, p.b.size(), fp);
}

// vtk_writer_write(particle_gpu*) (vtk_writer.cpp:78-262), from the host snapshot
int write_particles(const OutputJob &J, std::string &err) {
    const int n = J.n;
    const float4 *S = J.h_snap;
    auto at = [&](int k, int i) -> const float4 & { return S[size_t(k) * n + i]; };
    std::vector<int> keep;
    keep.reserve(n);
    for (int i = 0; i < n; i++)
        if (at(SN_FT, i).w != 1.f) keep.push_back(i);
    const int m = int(keep.size());
    FILE *fp = fopen(J.path.c_str(), "w+");
    if (!fp) {
        err = "cannot open " + J.path;
        return MFREE_ERR_IO;
    }
    fprintf(fp, "# vtk DataFile Version 2.0\n");
    fprintf(fp, "mfree iwf\n");
    fprintf(fp, "ASCII\n");
    fprintf(fp, "\n");
    fprintf(fp, "DATASET UNSTRUCTURED_GRID\n");
    fprintf(fp, "POINTS %d float\n", m);
    sections(fp, m, [&](Text &t, int k) {
        const float4 &p = at(SN_POS, keep[k]);
        t.add("%f %f %f\n", p.x, p.y, p.z);
    });
    fprintf(fp, "\n");
    fprintf(fp, "CELLS %d %d\n", m, 2 * m);
    sections(fp, m, [&](Text &t, int k) { t.add("%d %d\n", 1, keep[k]); });
    fprintf(fp, "\n");
    fprintf(fp, "CELL_TYPES %d\n", m);
    sections(fp, m, [&](Text &t, int) { t.add("%d\n", 1); });
    fprintf(fp, "\n");
    fprintf(fp, "POINT_DATA %d\n", m);
    auto scalar = [&](const char *name, auto &&val) {
        fprintf(fp, "SCALARS %s float 1\n", name);
        fprintf(fp, "LOOKUP_TABLE default\n");
        sections(fp, m, [&](Text &t, int k) { t.add("%f\n", double(val(keep[k]))); });
        fprintf(fp, "\n");
    };
    scalar("density", [&](int i) { return at(SN_VEL, i).w; });
    scalar("contact", [&](int i) {
        const float4 &f = at(SN_FC, i);
        return std::sqrt(f.x * f.x + f.y * f.y + f.z * f.z) > 0.f ? 1.0 : 0.0;
    });
    scalar("Temperature", [&](int i) { return at(SN_SB, i).z; });
    scalar("Fixed", [&](int i) { return at(SN_DSB, i).w; });
    scalar("Tool", [&](int i) { return at(SN_FC, i).w; });
    scalar("EquivAccumPlasticStrain", [&](int i) { return at(SN_SB, i).w; });
    scalar("Svm", [&](int i) {
        // pressure of the last half step (do_material_eos), zero for tool particles
        const float p = at(SN_FC, i).w == 1.f ? 0.f : J.c0sq * (at(SN_RV, i).w - J.rho0);
        const float4 &a = at(SN_SA, i), &b = at(SN_SB, i);
        const double sxx = a.x - p, syy = a.y - p, szz = a.z - p;
        const double sxy = a.w, sxz = b.x, syz = b.y;
        const double s2 = (sxx * sxx + syy * syy + szz * szz) - sxx * syy - sxx * szz - syy * szz +
                          3.0 * (sxy * sxy + syz * syz + sxz * sxz);
        return s2 > 0 ? std::sqrt(s2) : 0.;
    });
    const bool bad = ferror(fp) != 0;
    fclose(fp);
    if (bad) {
        err = "write error on " + J.path;
        return MFREE_ERR_IO;
    }
    return MFREE_OK;
}

int ensure_job(mfree_ctx *c) {
    if (c->output && c->output->n == c->n_init) return MFREE_OK;
    finish_output(c, true);
    auto *J = new OutputJob();
    c->output = J;
    J->device = c->device;
    J->n = c->n_init;
    const size_t bytes = sizeof(float4) * SN_N * size_t(c->n_init);
    CUDA_TRY(cudaStreamCreateWithFlags(&J->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&J->snap, cudaEventDisableTiming));
    CUDA_TRY(cudaMalloc(&J->d_snap, bytes));
    c->bytes += bytes;  // (finish_output subtracts it again with the buffer)
    CUDA_TRY(cudaMallocHost(&J->h_snap, bytes));
    return MFREE_OK;
}

float current_time(const mfree_ctx *c) { return c->t; }  // the time of the last step (tool and box positions)

}  // namespace

int mfree::host::finish_output(mfree_ctx *c, bool release) {
    OutputJob *J = c->output;
    if (!J) return MFREE_OK;
    if (J->worker.joinable()) J->worker.join();
    int st = J->status;
    if (st) fail(st, J->err);
    J->status = MFREE_OK;
    if (release) {
        if (J->stream) cudaStreamSynchronize(J->stream);
        if (J->d_snap) {
            cudaFree(J->d_snap);
            c->bytes -= sizeof(float4) * SN_N * size_t(J->n);
        }
        if (J->h_snap) cudaFreeHost(J->h_snap);
        if (J->snap) cudaEventDestroy(J->snap);
        if (J->stream) cudaStreamDestroy(J->stream);
        delete J;
        c->output = nullptr;
    }
    return st;
}

extern "C" {

int mfree_write_vtk(mfree_ctx *c, const char *path) {
    if (!c || !path) return fail(MFREE_ERR_ARG, "mfree_write_vtk: null argument");
    int st = finish_output(c, false);  // one output in flight
    if (st) return st;
    if ((st = ensure_job(c))) return st;
    OutputJob *J = c->output;
    const int n = c->n_init;
    const State &S = c->st[c->cur];
    const float4 *src[SN_N] = {S.pos4, S.vel4, S.sa4, S.sb4, S.dsb4, S.fc4, S.ft4, c->rec.f[REC_V]};
    for (int k = 0; k < SN_N; k++) {  // (the V records are interleaved with four others: a pitched copy)
        const size_t pitch = sizeof(float4) * (src[k] == c->rec.f[REC_V] ? rec_stride(REC_V) : 1);
        CUDA_TRY(cudaMemcpy2DAsync(J->d_snap + size_t(k) * n, sizeof(float4), src[k], pitch, sizeof(float4), n,
                                   cudaMemcpyDeviceToDevice, c->stream));
    }
    CUDA_TRY(cudaEventRecord(J->snap, c->stream));
    CUDA_TRY(cudaStreamWaitEvent(J->stream, J->snap, 0));
    CUDA_TRY(cudaMemcpyAsync(J->h_snap, J->d_snap, sizeof(float4) * SN_N * size_t(n), cudaMemcpyDeviceToHost,
                             J->stream));
    const float c0 = std::sqrt(c->phys.rho0 != 0.f ? c->phys.K / c->phys.rho0 : 0.f);
    J->c0sq = c0 * c0;
    J->rho0 = c->phys.rho0;
    J->path = path;
    J->worker = std::thread([J] {
        cudaSetDevice(J->device);
        cudaError_t e = cudaStreamSynchronize(J->stream);
        if (e != cudaSuccess) {
            J->status = MFREE_ERR_CUDA;
            J->err = std::string("mfree_write_vtk copy: ") + cudaGetErrorString(e);
            return;
        }
        J->status = write_particles(*J, J->err);
    });
    return MFREE_OK;
}

int mfree_output_wait(mfree_ctx *c) {
    if (!c) return fail(MFREE_ERR_ARG, "mfree_output_wait: null context");
    return finish_output(c, false);
}

int mfree_write_vtk_tools(mfree_ctx *c, const char *path) {
    if (!c || !path) return fail(MFREE_ERR_ARG, "mfree_write_vtk_tools: null argument");
    const float t = current_time(c);
    size_t npos = 0, ntri = 0;
    for (auto &tp : c->tools) {
        npos += tp->verts.size() / 3;
        ntri += tp->host.tris.size();
    }
    FILE *fp = fopen(path, "w+");
    if (!fp) return fail(MFREE_ERR_IO, std::string("cannot open ") + path);
    fprintf(fp, "# vtk DataFile Version 2.0\n");
    fprintf(fp, "mfree iwf\n");
    fprintf(fp, "ASCII\n");
    fprintf(fp, "\n");
    fprintf(fp, "DATASET UNSTRUCTURED_GRID\n");
    fprintf(fp, "POINTS %d float\n", int(npos));
    for (auto &tp : c->tools)  // p_init + v t, as the contact uses them
        for (size_t v = 0; v + 2 < tp->verts.size(); v += 3)
            fprintf(fp, "%f %f %f\n", double(tp->verts[v] + tp->vel[0] * t), double(tp->verts[v + 1] + tp->vel[1] * t),
                    double(tp->verts[v + 2] + tp->vel[2] * t));
    fprintf(fp, "\n");
    fprintf(fp, "CELLS %d %d\n", int(ntri), int(3 * ntri + ntri));
    int offset = 0;
    for (auto &tp : c->tools) {
        for (auto &tr : tp->host.tris) fprintf(fp, "%d %d %d %d\n", 3, tr.i1 + offset, tr.i2 + offset, tr.i3 + offset);
        offset += int(tp->verts.size() / 3);
    }
    fprintf(fp, "\n");
    fprintf(fp, "CELL_TYPES %d\n", int(ntri));
    for (auto &tp : c->tools)
        for (size_t k = 0; k < tp->host.tris.size(); k++) fprintf(fp, "%d\n", 5);
    fprintf(fp, "POINT_DATA %d\n", int(npos));
    fprintf(fp, "SCALARS id float 1\n");
    fprintf(fp, "LOOKUP_TABLE default\n");
    for (size_t k = 0; k < c->tools.size(); k++)
        for (size_t v = 0; v < c->tools[k]->verts.size() / 3; v++) fprintf(fp, "%d\n", int(k));
    fprintf(fp, "\n");
    fprintf(fp, "SCALARS active float 1\n");
    fprintf(fp, "LOOKUP_TABLE default\n");
    for (auto &tp : c->tools) {
        const int alive = (t >= tp->birth && t <= tp->death) ? 1 : 0;
        for (size_t v = 0; v < tp->verts.size() / 3; v++) fprintf(fp, "%d\n", alive);
    }
    fprintf(fp, "\n");
    const bool bad = ferror(fp) != 0;
    fclose(fp);
    return bad ? fail(MFREE_ERR_IO, std::string("write error on ") + path) : MFREE_OK;
}

int mfree_write_vtk_blanking(mfree_ctx *c, const char *path) {
    if (!c || !path) return fail(MFREE_ERR_ARG, "mfree_write_vtk_blanking: null argument");
    if (!c->blank_set) return fail(MFREE_ERR_ARG, "mfree_write_vtk_blanking: no blanking box");
    const float t = current_time(c);
    float lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        lo[d] = c->b_min[d] + t * c->b_vel[d];
        hi[d] = c->b_max[d] + t * c->b_vel[d];
    }
    // corners 000, 100, 110, 010, 001, 101, 111, 011
    const float cx[8] = {lo[0], hi[0], hi[0], lo[0], lo[0], hi[0], hi[0], lo[0]};
    const float cy[8] = {lo[1], lo[1], hi[1], hi[1], lo[1], lo[1], hi[1], hi[1]};
    const float cz[8] = {lo[2], lo[2], lo[2], lo[2], hi[2], hi[2], hi[2], hi[2]};
    FILE *fp = fopen(path, "w+");
    if (!fp) return fail(MFREE_ERR_IO, std::string("cannot open ") + path);
    fprintf(fp, "# vtk DataFile Version 2.0\n");
    fprintf(fp, "mfree iwf\n");
    fprintf(fp, "ASCII\n");
    fprintf(fp, "\n");
    fprintf(fp, "DATASET UNSTRUCTURED_GRID\n");
    fprintf(fp, "POINTS %d float\n", 8);
    for (int k = 0; k < 8; k++) fprintf(fp, "%f %f %f\n", double(cx[k]), double(cy[k]), double(cz[k]));
    fprintf(fp, "\n");
    fprintf(fp, "CELL_TYPES %d\n", 6);
    for (int k = 0; k < 6; k++) fprintf(fp, "%d\n", 9);
    fprintf(fp, "\n");
    static const int quad[6][4] = {{0, 1, 2, 3}, {0, 1, 5, 4}, {1, 2, 6, 5}, {0, 3, 7, 4}, {3, 2, 6, 7}, {4, 5, 6, 7}};
    fprintf(fp, "CELLS %d %d\n", 6, 5 * 6);
    for (auto &q : quad) fprintf(fp, "4 %d %d %d %d\n", q[0], q[1], q[2], q[3]);
    fprintf(fp, "\n");
    const bool bad = ferror(fp) != 0;
    fclose(fp);
    return bad ? fail(MFREE_ERR_IO, std::string("write error on ") + path) : MFREE_OK;
}

int mfree_append_force_log(mfree_ctx *c, const char *path) {
    if (!c || !path) return fail(MFREE_ERR_ARG, "mfree_append_force_log: null argument");
    std::vector<float> f(3 * std::max<size_t>(c->tools.size(), 1));
    if (!c->tools.empty()) {
        CUDA_TRY(cudaMemcpyAsync(f.data(), c->d_forces, sizeof(float) * 3 * c->tools.size(), cudaMemcpyDeviceToHost,
                                 c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
    FILE *fp = fopen(path, "a");
    if (!fp) return fail(MFREE_ERR_IO, std::string("cannot open ") + path);
    for (size_t k = 0; k < c->tools.size(); k++)
        fprintf(fp, "%.9g %.9g %.9g ", double(f[3 * k]), double(f[3 * k + 1]), double(f[3 * k + 2]));
    fprintf(fp, "\n");
    const bool bad = ferror(fp) != 0;
    fclose(fp);
    return bad ? fail(MFREE_ERR_IO, std::string("write error on ") + path) : MFREE_OK;
}

}  // extern "C"
