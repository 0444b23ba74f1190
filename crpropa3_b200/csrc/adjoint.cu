// adjoint.cu -- reverse-mode derivative of the fixed-step Boris push over a
// Grid3f (no reference counterpart; the forward step is
// PropagationBP::dY, PropagationBP.cpp:19, with the grid values taken as
// doubles and double trilinear weights in the corner order of Grid.h:571,
// then the direction normalised).
//
// Loss: L = sum_i (1 - u_final,i . target_i).  Gradients with respect to the
// initial directions, the energies and every grid value.
//
// One thread per candidate.  The forward pass stores the state (x, u) every
// K steps (checkpoints, FP64, in the caller's workspace).  The reverse pass
// walks the segments backwards: it recomputes one segment's K states from its
// checkpoint into thread-local memory and applies the adjoint of each step
// (normalisation, second half drift, Boris rotation, rotation vectors,
// field interpolation, first half drift).  The grid gradient is scattered
// with 64-bit integer atomics on fixed-point values (scale 2^36 / max kappa,
// kappa = q h c / 2E): integer addition is associative, so the result does
// not depend on the order the atomics land in.  Divisions are reciprocal
// multiplies and multiply-adds are contracted, so results agree with the
// oracle's CPU adjoint (which divides) to rounding, not bit for bit.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "crp_gpu.h"
#include "engine_internal.h"

namespace crp {
void set_last_error(const char *msg);
}

using namespace crp;

namespace {

constexpr int kMaxK = 128;
constexpr double kC = 2.99792458e8;

struct v3 { double x, y, z; };
__device__ __forceinline__ v3 mk(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ v3 add(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 sub(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 muls(v3 a, double f) { return {a.x * f, a.y * f, a.z * f}; }
__device__ __forceinline__ v3 divs(v3 a, double f) { return {a.x / f, a.y / f, a.z / f}; }
__device__ __forceinline__ double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 cross(v3 a, v3 v) {
    return {a.y * v.z - v.y * a.z, a.z * v.x - v.z * a.x, a.x * v.y - v.x * a.y};
}
__device__ __forceinline__ double norm(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

struct AdjGrid {
    const float *g;
    int nx, ny, nz;
    bool pow2;  // every dimension a power of two: indices wrap with a mask
    double gox, goy, goz, sx, sy, sz;
    double isx, isy, isz;  // 1 / spacing
};

// periodic index: i mod n in [0, n) (a mask for power-of-two n, the same value)
__device__ __forceinline__ int wrap_index(int i, int n, bool pow2) {
    return pow2 ? (i & (n - 1)) : ((i % n) + n) % n;
}

// corner indices, weights and weight gradients of the cell around x
__device__ __forceinline__ void cell(const AdjGrid &G, v3 x, size_t idx[8], double w[8], double dw[8][3]) {
    const double r[3] = {(x.x - G.gox) * G.isx, (x.y - G.goy) * G.isy, (x.z - G.goz) * G.isz};
    const int n[3] = {G.nx, G.ny, G.nz};
    const double is[3] = {G.isx, G.isy, G.isz};
    int lo[3], hi[3];
    double f0[3], f1[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        double fl = floor(r[a]);
        lo[a] = wrap_index((int)fl, n[a], G.pow2);
        hi[a] = G.pow2 ? (lo[a] + 1) & (n[a] - 1) : (lo[a] + 1) % n[a];
        f0[a] = r[a] - fl;
        f1[a] = 1 - f0[a];
    }
    const int sel[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 0}, {1, 1, 1}};
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int ix = sel[k][0] ? hi[0] : lo[0], iy = sel[k][1] ? hi[1] : lo[1], iz = sel[k][2] ? hi[2] : lo[2];
        idx[k] = ((size_t)ix * G.ny + (size_t)iy) * G.nz + (size_t)iz;
        const double wx = sel[k][0] ? f0[0] : f1[0], wy = sel[k][1] ? f0[1] : f1[1], wz = sel[k][2] ? f0[2] : f1[2];
        const double sx = sel[k][0] ? is[0] : -is[0], sy = sel[k][1] ? is[1] : -is[1],
                     sz = sel[k][2] ? is[2] : -is[2];
        w[k] = wx * wy * wz;
        dw[k][0] = sx * wy * wz;
        dw[k][1] = wx * sy * wz;
        dw[k][2] = wx * wy * sz;
    }
}

__device__ __forceinline__ v3 field(const AdjGrid &G, const size_t idx[8], const double w[8]) {
    v3 B = mk(0, 0, 0);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const float *c = G.g + 3 * idx[k];
        B.x += w[k] * (double)__ldg(c);
        B.y += w[k] * (double)__ldg(c + 1);
        B.z += w[k] * (double)__ldg(c + 2);
    }
    return B;
}

__device__ __forceinline__ void step(const AdjGrid &G, v3 &x, v3 &u, double hh, double kappa) {
    v3 x1 = add(x, muls(u, hh));
    size_t idx[8];
    double w[8], dw[8][3];
    cell(G, x1, idx, w, dw);
    v3 B = field(G, idx, w);
    v3 t = muls(B, kappa);
    double D = 1 + dot(t, t);
    v3 s = muls(t, 2 * (1 / D));
    v3 v = add(u, cross(u, t));
    v3 u2 = add(u, cross(v, s));
    x = add(x1, muls(u2, hh));
    u = muls(u2, 1 / norm(u2));
}

struct IO {
    uint64_t n;
    const double *x, *y, *z, *dx, *dy, *dz, *energy, *charge, *tx, *ty, *tz;
    double *loss, *ux, *uy, *uz, *gdx, *gdy, *gdz, *ge;
};

__global__ void kappa_max_kernel(IO io, double h, unsigned long long *kmax) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double k = 0;
    if (i < io.n) k = fabs(io.charge[i] * h * kC / (2 * io.energy[i]));
    unsigned long long b = __double_as_longlong(k);  // non-negative doubles order as integers
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long ob = __shfl_xor_sync(0xffffffffu, b, o);
        b = ob > b ? ob : b;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(kmax, b);
}

// forward pass; with ckpt != null the state before every K-th step is stored
__global__ void __launch_bounds__(128) forward_kernel(AdjGrid G, IO io, double h, int n_steps, int K,
                                                      double *ckpt) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= io.n) return;
    const double kappa = io.charge[i] * h * kC / (2 * io.energy[i]);
    const double hh = h / 2;
    v3 x = mk(io.x[i], io.y[i], io.z[i]), u = mk(io.dx[i], io.dy[i], io.dz[i]);
    const uint64_t n = io.n;
    for (int k = 0; k < n_steps; k++) {
        if (ckpt && k % K == 0) {
            double *c = ckpt + (size_t)(k / K) * 6 * n;
            c[i] = x.x; c[n + i] = x.y; c[2 * n + i] = x.z;
            c[3 * n + i] = u.x; c[4 * n + i] = u.y; c[5 * n + i] = u.z;
        }
        step(G, x, u, hh, kappa);
    }
    io.loss[i] = 1 - dot(u, mk(io.tx[i], io.ty[i], io.tz[i]));
    if (io.ux) { io.ux[i] = u.x; io.uy[i] = u.y; io.uz[i] = u.z; }
}

// Cell of the periodic grid around x: per-axis lower / upper indices and the
// linear fractions (corner weights and their gradients are formed from these
// on the fly, which keeps the reverse kernel's registers in budget).
struct CellW {
    int lo[3], hi[3];
    double f0[3], f1[3];
};

__device__ __forceinline__ CellW cellw(const AdjGrid &G, v3 x) {
    CellW c;
    const double r[3] = {(x.x - G.gox) * G.isx, (x.y - G.goy) * G.isy, (x.z - G.goz) * G.isz};
    const int n[3] = {G.nx, G.ny, G.nz};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double fl = floor(r[a]);
        c.lo[a] = wrap_index((int)fl, n[a], G.pow2);
        c.hi[a] = G.pow2 ? (c.lo[a] + 1) & (n[a] - 1) : (c.lo[a] + 1) % n[a];
        c.f0[a] = r[a] - fl;
        c.f1[a] = 1 - c.f0[a];
    }
    return c;
}

// corner q of the Grid.h:571 order: which of lo / hi on each axis
__device__ __forceinline__ int bit(int q, int a) {
    const int t[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 0}, {1, 1, 1}};
    return t[q][a];
}

__device__ __forceinline__ size_t corner_index(const AdjGrid &G, const int lo[3], const int hi[3], int q) {
    const int ix = bit(q, 0) ? hi[0] : lo[0], iy = bit(q, 1) ? hi[1] : lo[1], iz = bit(q, 2) ? hi[2] : lo[2];
    return ((size_t)ix * G.ny + (size_t)iy) * G.nz + (size_t)iz;
}

// add one cell's summed contributions to the fixed-point accumulator
__device__ __forceinline__ void flush(const AdjGrid &G, unsigned long long *acc, const int lo[3],
                                      const int hi[3], double g[8][3], double scale) {
    if (lo[0] >= 0) {
#pragma unroll
        for (int q = 0; q < 8; q++) {
            unsigned long long *a = acc + 3 * corner_index(G, lo, hi, q);
            atomicAdd(a, (unsigned long long)__double2ll_rn(g[q][0] * scale));
            atomicAdd(a + 1, (unsigned long long)__double2ll_rn(g[q][1] * scale));
            atomicAdd(a + 2, (unsigned long long)__double2ll_rn(g[q][2] * scale));
        }
    }
#pragma unroll
    for (int q = 0; q < 8; q++) g[q][0] = g[q][1] = g[q][2] = 0;
}

__global__ void __launch_bounds__(128, 2) reverse_kernel(AdjGrid G, IO io, double h, int n_steps, int K,
                                                      const double *ckpt,
                                                      unsigned long long *acc,
                                                      const unsigned long long *kmax_bits) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= io.n) return;
    const uint64_t n = io.n;
    const double kappa = io.charge[i] * h * kC / (2 * io.energy[i]);
    const double hh = h / 2;
    const double kmax = __longlong_as_double((long long)*kmax_bits);
    const double scale = (acc && kmax > 0) ? ldexp(1.0 / kmax, 36) : 0.0;
    const double is[3] = {G.isx, G.isy, G.isz};
    v3 xs[kMaxK], us[kMaxK];
    v3 xb = mk(0, 0, 0), ub = mk(-io.tx[i], -io.ty[i], -io.tz[i]);
    double kb = 0;
    // the cell the candidate is in: its corner values, and its grid-gradient
    // contributions summed in registers and flushed with atomics when the
    // candidate leaves the cell
    int clo[3] = {-1, -1, -1}, chi[3] = {-1, -1, -1};
    float gc[8][3];
    double gacc[8][3];
#pragma unroll
    for (int q = 0; q < 8; q++) gacc[q][0] = gacc[q][1] = gacc[q][2] = 0;
    const int nseg = (n_steps + K - 1) / K;
    for (int j = nseg - 1; j >= 0; j--) {
        const double *c = ckpt + (size_t)j * 6 * n;
        const int k0 = j * K, k1 = (k0 + K < n_steps) ? k0 + K : n_steps;
        v3 x = mk(c[i], c[n + i], c[2 * n + i]), u = mk(c[3 * n + i], c[4 * n + i], c[5 * n + i]);
        // the states before each step of the segment (the segment's own end
        // state is not needed: checkpoint_every = 1 recomputes nothing)
        for (int k = k0; k < k1; k++) {
            xs[k - k0] = x; us[k - k0] = u;
            if (k + 1 < k1) step(G, x, u, hh, kappa);
        }
        for (int k = k1 - 1; k >= k0; k--) {
            const v3 u0 = us[k - k0];
            const v3 x1 = add(xs[k - k0], muls(u0, hh));
            const CellW cw = cellw(G, x1);
            // a new cell: flush the previous cell's gradient, load this one's corners
            // (a candidate stays in one cell for several steps)
            if (cw.lo[0] != clo[0] || cw.lo[1] != clo[1] || cw.lo[2] != clo[2] || cw.hi[0] != chi[0] ||
                cw.hi[1] != chi[1] || cw.hi[2] != chi[2]) {
                if (acc) flush(G, acc, clo, chi, gacc, scale);
#pragma unroll
                for (int a = 0; a < 3; a++) { clo[a] = cw.lo[a]; chi[a] = cw.hi[a]; }
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const float *cg = G.g + 3 * corner_index(G, cw.lo, cw.hi, q);
                    gc[q][0] = __ldg(cg); gc[q][1] = __ldg(cg + 1); gc[q][2] = __ldg(cg + 2);
                }
            }
            v3 B = mk(0, 0, 0);
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const double wq = (bit(q, 0) ? cw.f0[0] : cw.f1[0]) * (bit(q, 1) ? cw.f0[1] : cw.f1[1]) *
                                  (bit(q, 2) ? cw.f0[2] : cw.f1[2]);
                B.x += wq * (double)gc[q][0];
                B.y += wq * (double)gc[q][1];
                B.z += wq * (double)gc[q][2];
            }
            const v3 t = muls(B, kappa);
            const double D = 1 + dot(t, t);
            const double iD = 1 / D;
            const v3 s = muls(t, 2 * iD);
            const v3 v = add(u0, cross(u0, t));
            const v3 u2 = add(u0, cross(v, s));
            const double inn = 1 / norm(u2);
            const v3 un = muls(u2, inn);
            // reverse of: normalisation, second half drift, Boris rotation
            v3 u2b = muls(sub(ub, muls(un, dot(un, ub))), inn);
            u2b = add(u2b, muls(xb, hh));
            const v3 vb = cross(s, u2b);
            const v3 sb = cross(u2b, v);
            const v3 ubar = add(u2b, add(vb, cross(t, vb)));
            v3 tb = cross(vb, u0);
            tb = add(tb, sub(muls(sb, 2 * iD), muls(t, 4 * dot(t, sb) * (iD * iD))));
            const v3 Bb = muls(tb, kappa);
            kb += dot(tb, B);
            // reverse of the interpolation: position Jacobian and grid values
            v3 x1b = xb;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const double wx = bit(q, 0) ? cw.f0[0] : cw.f1[0], wy = bit(q, 1) ? cw.f0[1] : cw.f1[1],
                             wz = bit(q, 2) ? cw.f0[2] : cw.f1[2];
                const double sx = bit(q, 0) ? is[0] : -is[0], sy = bit(q, 1) ? is[1] : -is[1],
                             sz = bit(q, 2) ? is[2] : -is[2];
                const double gdot = Bb.x * (double)gc[q][0] + Bb.y * (double)gc[q][1] + Bb.z * (double)gc[q][2];
                x1b.x += gdot * (sx * wy * wz);
                x1b.y += gdot * (wx * sy * wz);
                x1b.z += gdot * (wx * wy * sz);
                const double wq = wx * wy * wz;
                gacc[q][0] += wq * Bb.x;
                gacc[q][1] += wq * Bb.y;
                gacc[q][2] += wq * Bb.z;
            }
            xb = x1b;
            ub = add(ubar, muls(x1b, hh));
        }
    }
    if (acc) flush(G, acc, clo, chi, gacc, scale);
    io.gdx[i] = ub.x; io.gdy[i] = ub.y; io.gdz[i] = ub.z;
    io.ge[i] = kb * (-kappa / io.energy[i]);
}

__global__ void finalize_kernel(const unsigned long long *acc, uint64_t m,
                                const unsigned long long *kmax_bits, double *out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const double kmax = __longlong_as_double((long long)*kmax_bits);
    out[i] = (double)(long long)acc[i] * ldexp(kmax, -36);
}

crp_status fail(crp_status st, const char *msg) {
    set_last_error(msg);
    return st;
}

crp_status cuda_fail(cudaError_t e, const char *what) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    set_last_error(buf);
    return e == cudaErrorMemoryAllocation ? CRP_ERR_OUT_OF_MEMORY : CRP_ERR_CUDA;
}

crp_status check_desc(const crp_adjoint_desc *d, const crp_adjoint_io *io) {
    if (!d || !io) return fail(CRP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!d->grid_values || !d->nx || !d->ny || !d->nz) return fail(CRP_ERR_INVALID_ARGUMENT, "Grid3f: empty grid");
    if (d->nx > (1u << 20) || d->ny > (1u << 20) || d->nz > (1u << 20))
        return fail(CRP_ERR_CAPACITY, "Grid3f: a dimension beyond 2^20 cells");
    if (!(d->step > 0)) return fail(CRP_ERR_INVALID_ARGUMENT, "step must be > 0");
    if (d->n_steps < 0) return fail(CRP_ERR_INVALID_ARGUMENT, "n_steps < 0");
    if (d->checkpoint_every < 1 || d->checkpoint_every > kMaxK)
        return fail(CRP_ERR_CAPACITY, "checkpoint_every must be 1..128");
    if (io->n && (!io->x || !io->y || !io->z || !io->dx || !io->dy || !io->dz || !io->energy ||
                  !io->charge || !io->tx || !io->ty || !io->tz || !io->loss))
        return fail(CRP_ERR_INVALID_ARGUMENT, "an input array is NULL");
    return CRP_OK;
}

AdjGrid make_grid(const crp_adjoint_desc *d) {
    AdjGrid G;
    G.g = d->grid_values;
    G.nx = (int)d->nx; G.ny = (int)d->ny; G.nz = (int)d->nz;
    auto p2 = [](uint64_t v) { return v && !(v & (v - 1)); };
    G.pow2 = p2(d->nx) && p2(d->ny) && p2(d->nz);
    G.gox = d->origin[0] + d->spacing[0] / 2;
    G.goy = d->origin[1] + d->spacing[1] / 2;
    G.goz = d->origin[2] + d->spacing[2] / 2;
    G.sx = d->spacing[0]; G.sy = d->spacing[1]; G.sz = d->spacing[2];
    G.isx = 1.0 / G.sx; G.isy = 1.0 / G.sy; G.isz = 1.0 / G.sz;
    return G;
}

IO make_io(const crp_adjoint_io *a) {
    IO io;
    io.n = a->n;
    io.x = a->x; io.y = a->y; io.z = a->z; io.dx = a->dx; io.dy = a->dy; io.dz = a->dz;
    io.energy = a->energy; io.charge = a->charge; io.tx = a->tx; io.ty = a->ty; io.tz = a->tz;
    io.loss = a->loss; io.ux = a->ux; io.uy = a->uy; io.uz = a->uz;
    io.gdx = a->grad_dx; io.gdy = a->grad_dy; io.gdz = a->grad_dz; io.ge = a->grad_energy;
    return io;
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

extern "C" {

crp_status crp_bp_adjoint_workspace(const crp_adjoint_desc *d, uint64_t n, size_t *bytes) {
    if (!d || !bytes) return fail(CRP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (d->checkpoint_every < 1 || d->checkpoint_every > kMaxK)
        return fail(CRP_ERR_CAPACITY, "checkpoint_every must be 1..128");
    const size_t nck = (size_t)((d->n_steps + d->checkpoint_every - 1) / d->checkpoint_every);
    *bytes = align256(256) + align256(nck * 6 * n * sizeof(double)) +
             align256((size_t)d->nx * d->ny * d->nz * 3 * sizeof(unsigned long long));
    return CRP_OK;
}

crp_status crp_bp_forward_loss(const crp_adjoint_desc *d, const crp_adjoint_io *a, void *stream) {
    crp_status st = check_desc(d, a);
    if (st) return st;
    if (a->n == 0) return CRP_OK;
    forward_kernel<<<(unsigned)((a->n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        make_grid(d), make_io(a), d->step, d->n_steps, d->checkpoint_every, nullptr);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CRP_OK : cuda_fail(e, "adjoint forward kernel launch");
}

static crp_status adjoint_impl(const crp_adjoint_desc *d, const crp_adjoint_io *a, void *workspace,
                               size_t workspace_bytes, void *stream, bool do_forward,
                               bool do_backward) {
    crp_status st = check_desc(d, a);
    if (st) return st;
    if (do_backward && (!a->grad_dx || !a->grad_dy || !a->grad_dz || !a->grad_energy))
        return fail(CRP_ERR_INVALID_ARGUMENT, "a gradient array is NULL");
    size_t need = 0;
    st = crp_bp_adjoint_workspace(d, a->n, &need);
    if (st) return st;
    if (!workspace || workspace_bytes < need) return fail(CRP_ERR_CAPACITY, "workspace smaller than crp_bp_adjoint_workspace");
    if (a->n == 0) return CRP_OK;
    cudaStream_t s = (cudaStream_t)stream;
    char *w = static_cast<char *>(workspace);
    unsigned long long *kmax = reinterpret_cast<unsigned long long *>(w);
    const size_t nck = (size_t)((d->n_steps + d->checkpoint_every - 1) / d->checkpoint_every);
    double *ckpt = reinterpret_cast<double *>(w + align256(256));
    const size_t cells3 = (size_t)d->nx * d->ny * d->nz * 3;
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(w + align256(256) + align256(nck * 6 * a->n * sizeof(double)));
    const AdjGrid G = make_grid(d);
    const IO io = make_io(a);
    const unsigned blocks = (unsigned)((a->n + 127) / 128);
    cudaError_t e = cudaSuccess;
    if (do_forward) {
        e = cudaMemsetAsync(kmax, 0, 8, s);
        if (e != cudaSuccess) return cuda_fail(e, "clearing the adjoint workspace");
        kappa_max_kernel<<<blocks, 128, 0, s>>>(io, d->step, kmax);
        forward_kernel<<<blocks, 128, 0, s>>>(G, io, d->step, d->n_steps, d->checkpoint_every, ckpt);
    }
    if (do_backward) {
        if (a->grad_grid) {
            e = cudaMemsetAsync(acc, 0, cells3 * sizeof(unsigned long long), s);
            if (e != cudaSuccess) return cuda_fail(e, "clearing the adjoint workspace");
        }
        reverse_kernel<<<blocks, 128, 0, s>>>(G, io, d->step, d->n_steps, d->checkpoint_every, ckpt,
                                              a->grad_grid ? acc : nullptr, kmax);
        if (a->grad_grid)
            finalize_kernel<<<(unsigned)((cells3 + 255) / 256), 256, 0, s>>>(acc, cells3, kmax, a->grad_grid);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? CRP_OK : cuda_fail(e, "adjoint kernel launch");
}

crp_status crp_bp_adjoint(const crp_adjoint_desc *d, const crp_adjoint_io *a, void *workspace,
                          size_t workspace_bytes, void *stream) {
    return adjoint_impl(d, a, workspace, workspace_bytes, stream, true, true);
}

crp_status crp_bp_adjoint_forward(const crp_adjoint_desc *d, const crp_adjoint_io *a, void *workspace,
                                  size_t workspace_bytes, void *stream) {
    return adjoint_impl(d, a, workspace, workspace_bytes, stream, true, false);
}

crp_status crp_bp_adjoint_backward(const crp_adjoint_desc *d, const crp_adjoint_io *a, void *workspace,
                                   size_t workspace_bytes, void *stream) {
    return adjoint_impl(d, a, workspace, workspace_bytes, stream, false, true);
}

}  // extern "C"
