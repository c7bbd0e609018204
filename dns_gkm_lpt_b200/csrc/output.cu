// File output of the reference, written from the device state (declarations
// in include/gkm.h).  Host code only: each writer copies what it needs to the
// host, forms the reference's derived quantities with the reference's
// expressions, and prints with the reference's formats, so a file written
// here is the file the reference writes for the same state.
//
//   writeField        src/update.cpp:1324-1339  text, one line per interior cell
//   writeParticleData src/update.cpp:1341-1379  text, one line per particle; T file
//   WriteReInit       src/update.cpp:1381-1422  binary restart in the IC format
//
// Text formatting is split over host threads (a 256^3 field is 16.7 M lines);
// the chunks are written in order.
#include "gkm_handle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

using gkm_host::cuda_fail;
using gkm_host::fail;

namespace {

// copy of the current state, 5 x nt^3 (the stream is synchronised)
gkm_status download_state(gkm_handle* h, std::vector<double>& W)
{
    const size_t nt3 = (size_t)h->fc.nt3;
    W.resize(5 * nt3);
    const double* src = h->buf[h->parity];
    CK(h, cudaMemcpyAsync(W.data(), src, sizeof(double) * 5 * nt3, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return GKM_OK;
}

gkm_status read_clock(gkm_handle* h, gkm::DevClock* c)
{
    CK(h, cudaMemcpyAsync(c, h->clock, sizeof(gkm::DevClock), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return GKM_OK;
}

// formats items [0, count) with fmt_item(i, std::string&) on up to 32 threads
// and writes the text to f in item order
template <class F>
bool write_parallel(FILE* f, long long count, F fmt_item)
{
    unsigned nth = std::thread::hardware_concurrency();
    nth = std::max(1u, std::min(nth, 32u));
    if (count < 4096) nth = 1;
    const long long chunk = 1 << 16;
    for (long long base = 0; base < count; base += chunk * nth) {
        std::vector<std::string> out(nth);
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nth; t++) {
            const long long b = base + t * chunk, e = std::min(count, b + chunk);
            if (b >= e) break;
            pool.emplace_back([&, t, b, e]() {
                out[t].reserve((size_t)(e - b) * 128);
                for (long long i = b; i < e; i++) fmt_item(i, out[t]);
            });
        }
        for (auto& th : pool) th.join();
        for (auto& s : out)
            if (!s.empty() && std::fwrite(s.data(), 1, s.size(), f) != s.size()) return false;
    }
    return true;
}

void append(std::string& s, const char* fmt, double v)
{
    char b[64];
    const int n = std::snprintf(b, sizeof(b), fmt, v);
    s.append(b, (size_t)n);
}

}  // namespace

extern "C" {

gkm_status gkm_write_field(gkm_handle* h, const char* path)
{
    if (!h || !path) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    std::vector<double> W;
    gkm_status s = download_state(h, W);
    if (s != GKM_OK) return s;
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(h, GKM_ERR_ARG, std::string("cannot open ") + path);
    const int n = h->fc.n, nt = h->fc.nt;
    const size_t nt3 = (size_t)h->fc.nt3;
    const double gm1 = h->cfg.params.gam - 1;
    // FOR(j) FOR(i) FOR(k) over interior cells; den, u, v, w, p as generateSplines forms them
    const bool ok = write_parallel(f, (long long)n * n * n, [&](long long e, std::string& out) {
        const int j = (int)(e / ((long long)n * n)), i = (int)((e / n) % n), k = (int)(e % n);
        const size_t I = ((size_t)(j + 3) * nt + (i + 3)) * nt + (k + 3);
        const double den = W[I];
        const double u = W[nt3 + I] / den, v = W[2 * nt3 + I] / den, w = W[3 * nt3 + I] / den;
        const double Vsqr = u * u + v * v + w * w;
        const double p = (den * gm1) * (W[4 * nt3 + I] / den - 0.5 * Vsqr);
        char b[256];
        const int len = std::snprintf(b, sizeof(b), "%d %d %d %.15e %.15e %.15e %.15e %.15e\n", i, j, k, den, u, v, w, p);
        out.append(b, (size_t)len);
    });
    const bool closed = std::fclose(f) == 0;
    return ok && closed ? GKM_OK : fail(h, GKM_ERR_ARG, std::string("write failed: ") + path);
}

gkm_status gkm_write_reinit(gkm_handle* h, const char* path)
{
    if (!h || !path) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    std::vector<double> W;
    gkm_status s = download_state(h, W);
    if (s != GKM_OK) return s;
    const int n = h->fc.n, nt = h->fc.nt;
    const size_t nt3 = (size_t)h->fc.nt3, nc = (size_t)n * n * n;
    const double gm1 = h->cfg.params.gam - 1;
    std::vector<double> out(5 * nc);   // u0 | v0 | w0 | d0 | pr0, MATLAB (column-major) order
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++)
            for (int k = 0; k < n; k++) {
                const size_t I = ((size_t)(j + 3) * nt + (i + 3)) * nt + (k + 3);
                const size_t J = (size_t)k * n * n + (size_t)i * n + j;
                // c2p, src/update.cpp:844-853
                const double deni = W[I];
                const double ui = W[nt3 + I] / deni, vi = W[2 * nt3 + I] / deni, wi = W[3 * nt3 + I] / deni;
                const double Vsqr = (ui * ui + vi * vi + wi * wi);
                out[J] = ui;
                out[nc + J] = vi;
                out[2 * nc + J] = wi;
                out[3 * nc + J] = deni;
                out[4 * nc + J] = (deni * gm1) * (W[4 * nt3 + I] / deni - 0.5 * Vsqr);
            }
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(h, GKM_ERR_ARG, std::string("cannot open ") + path);
    const bool ok = std::fwrite(out.data(), sizeof(double), out.size(), f) == out.size();
    const bool closed = std::fclose(f) == 0;
    return ok && closed ? GKM_OK : fail(h, GKM_ERR_ARG, std::string("write failed: ") + path);
}

gkm_status gkm_write_particles(gkm_handle* h, const char* path)
{
    if (!h || !path) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    const int64_t np = h->np;
    std::vector<double> props((size_t)np * gkm::kPropCount), pos((size_t)np * 3);
    gkm_status s = gkm_host_props(h, props.data());
    if (s != GKM_OK) return s;
    if (np > 0) {
        s = gkm_particles_download(h, pos.data(), nullptr);
        if (s != GKM_OK) return s;
    }
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(h, GKM_ERR_ARG, std::string("cannot open ") + path);
    // column order of writeParticleData: x, y, z, then (x, y, z)-ordered vectors from the (y, x, z) table
    static const int cols[] = {0, 4, 5, 6, 16, 2, 1, 3, 8, 7, 9, 11, 10, 12, 14, 13, 15, 18, 17, 19,
                               33, 32, 34, 36, 35, 37, 39, 38, 40, 24, 23, 25, 21, 20, 22, 27, 26, 28};
    const int ncols = (int)(sizeof(cols) / sizeof(cols[0]));
    const bool ok = write_parallel(f, np, [&](long long p, std::string& out) {
        const double* P = props.data() + (size_t)p * gkm::kPropCount;
        char b[32];
        const int len = std::snprintf(b, sizeof(b), "%d ", (int)p);
        out.append(b, (size_t)len);
        append(out, "%.15e ", pos[3 * p + 1]);
        append(out, "%.15e ", pos[3 * p + 0]);
        append(out, "%.15e ", pos[3 * p + 2]);
        for (int c = 0; c < ncols; c++) append(out, c + 1 < ncols ? "%.15e " : "%.15e\n", P[cols[c]]);
    });
    const bool closed = std::fclose(f) == 0;
    return ok && closed ? GKM_OK : fail(h, GKM_ERR_ARG, std::string("write failed: ") + path);
}

gkm_status gkm_write_time(gkm_handle* h, const char* path)
{
    if (!h || !path) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    gkm::DevClock c;
    gkm_status s = read_clock(h, &c);
    if (s != GKM_OK) return s;
    // dt of the coming step: the fixed dt, or the CFL rule on the current state (src/update.cpp:1053)
    double dt = h->dt_fixed;
    if (!h->dt_fixed_mode) {
        double mw;
        const unsigned long long bits = c.wave[h->parity];
        std::memcpy(&mw, &bits, sizeof(mw));
        dt = h->fc.cfl * h->fc.dx / mw;
    }
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(h, GKM_ERR_ARG, std::string("cannot open ") + path);
    const bool ok = std::fprintf(f, "%.15e %.15e %.15e", c.t, dt, h->cfg.params.t0) > 0;
    const bool closed = std::fclose(f) == 0;
    return ok && closed ? GKM_OK : fail(h, GKM_ERR_ARG, std::string("write failed: ") + path);
}

}  // extern "C"
