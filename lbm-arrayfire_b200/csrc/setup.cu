// setup.cu — host-side helpers: descriptor defaults and validation, the reference drivers'
// loop-invariant set-up (masks and boundary classes), relaxation rules and MRT coefficients.
#include <cmath>
#include <cstring>

#include "internal.h"
#include "lattice.cuh"

namespace lbm {

static thread_local std::string g_error;

int set_error(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

int cuda_error(cudaError_t e, const char* what) {
    return set_error(LBM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

long long desc_cells(const lbm_desc* d) { return (long long)d->nx * d->ny * d->nz; }
int desc_q(const lbm_desc* d) { return d->lattice == LBM_D2Q9 ? 9 : 27; }
int storage_bytes(int storage) {
    switch (storage) {
        case LBM_F32: return 4;
        case LBM_F64: return 8;
        default: return 2;
    }
}
double default_scale(int storage) {
    // 2^14 lifts deviations down to ~4e-9 out of the FP16 subnormal range and still holds
    // deviations up to ~4 from the rest weight; BF16 has the FP32 exponent range and needs none.
    return storage == LBM_F16S ? 16384.0 : 1.0;
}

int validate_desc(const lbm_desc* d) {
    if (!d) return set_error(LBM_ERR_INVALID, "descriptor is NULL");
    if (d->lattice != LBM_D2Q9 && d->lattice != LBM_D3Q27)
        return set_error(LBM_ERR_INVALID, "lattice must be LBM_D2Q9 or LBM_D3Q27");
    if (d->collision < LBM_BGK || d->collision > LBM_SHANCHEN)
        return set_error(LBM_ERR_INVALID, "unknown collision");
    if (d->storage < LBM_F32 || d->storage > LBM_F64) return set_error(LBM_ERR_INVALID, "unknown storage");
    if (d->collision == LBM_MRT && d->lattice != LBM_D3Q27)
        return set_error(LBM_ERR_UNSUPPORTED, "MRT is built for D3Q27 only");
    if (d->collision == LBM_SHANCHEN && d->lattice != LBM_D2Q9)
        return set_error(LBM_ERR_UNSUPPORTED, "Shan-Chen is built for D2Q9 only");
    if (d->collision == LBM_MRT && d->mrt_basis != LBM_MRT_REF && d->mrt_basis != LBM_MRT_GRAM_SCHMIDT)
        return set_error(LBM_ERR_INVALID, "unknown MRT basis");
    if (d->arithmetic != LBM_ARITH_DEVIATION && d->arithmetic != LBM_ARITH_ABSOLUTE)
        return set_error(LBM_ERR_INVALID, "unknown arithmetic mode");
    if (d->rounding != LBM_ROUND_STOCHASTIC && d->rounding != LBM_ROUND_NEAREST)
        return set_error(LBM_ERR_INVALID, "unknown rounding mode");
    if (d->arithmetic == LBM_ARITH_ABSOLUTE && d->storage != LBM_F32 && d->storage != LBM_F64)
        return set_error(LBM_ERR_UNSUPPORTED, "absolute arithmetic needs F32 or F64 storage");
    if (d->arithmetic == LBM_ARITH_ABSOLUTE && d->collision == LBM_MRT)
        return set_error(LBM_ERR_UNSUPPORTED, "MRT runs in deviation arithmetic only");
    if (d->nx < 1 || d->ny < 1 || d->nz < 1) return set_error(LBM_ERR_INVALID, "lattice extents must be >= 1");
    if (d->lattice == LBM_D2Q9 && d->nz != 1) return set_error(LBM_ERR_INVALID, "D2Q9 needs nz == 1");
    if (d->nx > 0x7fffffffLL || d->ny > 65535 || d->nz > 65535)
        return set_error(LBM_ERR_INVALID, "extents beyond nx < 2^31, ny <= 65535, nz <= 65535");
    if (d->n_classes < 1 || d->n_classes > LBM_MAX_CLASSES)
        return set_error(LBM_ERR_INVALID, "n_classes must be in [1, 16]");
    if (!(d->omega > 0.0 && d->omega < 2.0) && d->collision != LBM_MRT)
        return set_error(LBM_ERR_INVALID, "omega must be in (0, 2)");
    if (d->storage_scale < 0.0) return set_error(LBM_ERR_INVALID, "storage_scale must be >= 0");
    if (d->storage_scale > 0.0) {
        int e;
        double m = std::frexp(d->storage_scale, &e);
        if (m != 0.5) return set_error(LBM_ERR_INVALID, "storage_scale must be a power of two");
    }
    for (int k = 0; k < d->n_classes; ++k) {
        const uint32_t fl = d->classes[k].flags;
        if (fl & ~0x1ffu) return set_error(LBM_ERR_INVALID, "unknown cell-class flag");
        if ((fl & (LBM_CELL_ZOUHE_VEL_XM | LBM_CELL_ZOUHE_RHO_XP)) &&
            (d->lattice != LBM_D2Q9 || d->collision != LBM_BGK))
            return set_error(LBM_ERR_UNSUPPORTED, "Zou-He boundaries are built for D2Q9 BGK only");
        if ((fl & LBM_CELL_ZOUHE_VEL_XM) && (fl & LBM_CELL_ZOUHE_RHO_XP))
            return set_error(LBM_ERR_INVALID, "a class is either a Zou-He inlet or a Zou-He outlet");
        if ((fl & LBM_CELL_ZOUHE_VEL_XM) && !(d->classes[k].ux < 1.0))
            return set_error(LBM_ERR_INVALID, "a Zou-He inlet needs ux < 1");
        if ((fl & LBM_CELL_ZOUHE_RHO_XP) && !(d->classes[k].rho > 0.0))
            return set_error(LBM_ERR_INVALID, "a Zou-He outlet needs rho > 0");
    }
    return LBM_OK;
}

// (X^-1 diag(v) X) for the 3x3 mix of the second-order diagonal slots.
static void mix_block(int basis, const double v[3], double dm, double out[9]) {
    const double Xr[9] = {1, 1, 1, 1, -1, 0, 1, 0, -1};
    const double Xg[9] = {1, 1, 1, 1, -1, 0, 1, 1, -2};
    const double* X = basis == kMrtRef ? Xr : Xg;
    // inverse by cofactors
    double inv[9];
    const double a = X[0], b = X[1], c = X[2], d = X[3], e = X[4], f = X[5], g = X[6], h = X[7], i = X[8];
    const double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
    inv[0] = (e * i - f * h) / det;
    inv[1] = (c * h - b * i) / det;
    inv[2] = (b * f - c * e) / det;
    inv[3] = (f * g - d * i) / det;
    inv[4] = (a * i - c * g) / det;
    inv[5] = (c * d - a * f) / det;
    inv[6] = (d * h - e * g) / det;
    inv[7] = (b * g - a * h) / det;
    inv[8] = (a * e - b * d) / det;
    for (int r = 0; r < 3; ++r)
        for (int col = 0; col < 3; ++col) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += inv[r * 3 + k] * v[k] * X[k * 3 + col];
            out[r * 3 + col] = dm * s;
        }
}

void mrt_coefficients(int basis, const double s[27], MrtCoef<double>& out) {
    for (int t = 0; t < 27; ++t) {
        const int row = mrt_slot_row(t);
        const double d = mrt_slot_scale(basis, t);
        if (row >= 0) {
            out.alpha[t] = d * (1.0 - s[row]);
            out.beta[t] = d * s[row];
        } else {
            out.alpha[t] = 0.0;
            out.beta[t] = 0.0;
        }
    }
    const double dm = mrt_slot_scale(basis, 2);
    const double keep[3] = {1.0 - s[7], 1.0 - s[8], 1.0 - s[9]};
    const double rate[3] = {s[7], s[8], s[9]};
    mix_block(basis, keep, dm, out.A);
    mix_block(basis, rate, dm, out.B);
}

}  // namespace lbm

using namespace lbm;

extern "C" {

int lbm_abi_version(void) { return LBM_ABI_VERSION; }

const char* lbm_last_error(void) { return g_error.c_str(); }

const char* lbm_strerror(int status) {
    switch (status) {
        case LBM_OK: return "ok";
        case LBM_ERR_INVALID: return "invalid argument";
        case LBM_ERR_CUDA: return "CUDA error";
        case LBM_ERR_NOMEM: return "out of memory";
        case LBM_ERR_DIVERGED: return "populations diverged (NaN/Inf)";
        case LBM_ERR_UNSUPPORTED: return "unsupported combination";
        case LBM_ERR_NO_DEVICE: return "no usable CUDA device";
        case LBM_ERR_STATE: return "invalid state for this call";
        case LBM_ERR_TIMEOUT: return "a bounded device-side wait timed out";
        default: return "unknown status";
    }
}

int lbm_q(int lattice) { return lattice == LBM_D2Q9 ? 9 : (lattice == LBM_D3Q27 ? 27 : 0); }

int lbm_velocities(int lattice, int32_t* cx, int32_t* cy, int32_t* cz, double* w, int32_t* opp) {
    const int q = lbm_q(lattice);
    if (!q) return set_error(LBM_ERR_INVALID, "unknown lattice");
    for (int i = 0; i < q; ++i) {
        const bool d2 = lattice == LBM_D2Q9;
        if (cx) cx[i] = d2 ? D2Q9::cx(i) : D3Q27::cx(i);
        if (cy) cy[i] = d2 ? D2Q9::cy(i) : D3Q27::cy(i);
        if (cz) cz[i] = d2 ? 0 : D3Q27::cz(i);
        if (w) w[i] = d2 ? D2Q9::w(i) : D3Q27::w(i);
        if (opp) opp[i] = d2 ? D2Q9::opp(i) : D3Q27::opp(i);
    }
    return LBM_OK;
}

void lbm_desc_init(lbm_desc* d, int lattice, int collision, int storage, int64_t nx, int64_t ny, int64_t nz) {
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    d->lattice = lattice;
    d->collision = collision;
    d->storage = storage;
    d->mrt_basis = LBM_MRT_REF;
    d->nx = nx;
    d->ny = ny;
    d->nz = nz;
    d->omega = 1.0;
    for (int i = 0; i < 27; ++i) d->mrt_s[i] = 1.0;
    d->sc_G = 0.0;
    d->storage_scale = 0.0;
    d->n_classes = 1;
    d->device = 0;
    d->classes[0].flags = 0;
    d->classes[0].rho = 1.0;
    d->mask = nullptr;
}

double lbm_omega_from_re(double u, double L, double re, int rule) {
    const double nu = rule == 1 ? u * 2.0 * L / re : u * L / re;
    return 1.0 / (3.0 * nu + 0.5);
}

void lbm_mrt_reference_rates(double s[27]) {
    // rust/examples/d3q27_mrt_lid.rs:111-150 (same values in cpp/d3q27_mrt_lid.cpp:97-137)
    const double s0 = 1.3, s1 = 1.3, sv = 1.1, sb = 0.9, s3 = 1.2, s3b = 0.9, s4 = 1.2, s4b = 1.2,
                 s5 = 1.1, s6 = 1.1;
    const double v[27] = {s0, s1, s1, s1, sv, sv, sv, sb, sv, sv, s3, s3, s3, s3,
                          s3, s3, s3b, s4, s4, s4, s4b, s4b, s4b, s5, s5, s5, s6};
    for (int i = 0; i < 27; ++i) s[i] = v[i];
}

void lbm_mrt_rates(double s[27], double sv, double other) {
    for (int i = 0; i < 27; ++i) s[i] = other;
    s[4] = s[5] = s[6] = s[8] = s[9] = sv;
}

static const uint32_t kSolidFlags = LBM_CELL_BOUNCE | LBM_CELL_SET_RHO | LBM_CELL_SET_UX | LBM_CELL_SET_UY |
                                    LBM_CELL_SET_UZ;

static void set_class(lbm_desc* d, int k, uint32_t flags, double rho, double ux, double uy, double uz) {
    d->classes[k].flags = flags;
    d->classes[k].reserved = 0;
    d->classes[k].rho = rho;
    d->classes[k].ux = ux;
    d->classes[k].uy = uy;
    d->classes[k].uz = uz;
}

int lbm_setup_cavity2d(lbm_desc* d, uint8_t* mask, double u_lid) {
    if (!d || !mask || d->lattice != LBM_D2Q9 || d->nx < 3 || d->ny < 2)
        return set_error(LBM_ERR_INVALID, "cavity2d needs a D2Q9 descriptor with nx >= 3, ny >= 2 and a mask");
    const int64_t nx = d->nx, ny = d->ny;
    // BOUND = 1; BOUND(1..nx-2, 1..ny-1) = 0  (cpp/d2q9_bgk_lid.cpp:90-91)
    for (int64_t y = 0; y < ny; ++y)
        for (int64_t x = 0; x < nx; ++x) {
            const bool fluid = x >= 1 && x <= nx - 2 && y >= 1;
            uint8_t k = fluid ? 0 : 1;
            if (fluid && y == ny - 1) k = 2;  // lid row: UX(lid, end), UY(lid, end) (:141-142)
            mask[x + nx * y] = k;
        }
    d->n_classes = 3;
    set_class(d, 0, 0, 1, 0, 0, 0);
    set_class(d, 1, kSolidFlags, 0, 0, 0, 0);  // UX(ON) = UY(ON) = DENSITY(ON) = 0 (:144-146)
    set_class(d, 2, LBM_CELL_SET_UX | LBM_CELL_SET_UY | LBM_CELL_SET_UZ, 1, u_lid, 0, 0);
    d->mask = mask;
    return LBM_OK;
}

int lbm_setup_cavity3d(lbm_desc* d, uint8_t* mask, double u_lid) {
    if (!d || !mask || d->lattice != LBM_D3Q27 || d->nx < 3 || d->ny < 3 || d->nz < 2)
        return set_error(LBM_ERR_INVALID, "cavity3d needs a D3Q27 descriptor with nx, ny >= 3, nz >= 2 and a mask");
    const int64_t nx = d->nx, ny = d->ny, nz = d->nz;
    // BOUND(1..nx-2, 1..ny-2, 1..nz-1) = 0 (cpp/d3q27_bgk_lid.cpp:119-120); lid plane z = nz-1 (:179-181)
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                const bool fluid = x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2 && z >= 1;
                uint8_t k = fluid ? 0 : 1;
                if (fluid && z == nz - 1) k = 2;
                mask[x + nx * (y + ny * z)] = k;
            }
    d->n_classes = 3;
    set_class(d, 0, 0, 1, 0, 0, 0);
    set_class(d, 1, kSolidFlags, 0, 0, 0, 0);
    set_class(d, 2, LBM_CELL_SET_UX | LBM_CELL_SET_UY | LBM_CELL_SET_UZ, 1, u_lid, 0, 0);
    d->mask = mask;
    return LBM_OK;
}

int lbm_setup_channel2d(lbm_desc* d, uint8_t* mask, double u_in, double ox, double oy, double r,
                        int config_mode) {
    if (!d || !mask || d->lattice != LBM_D2Q9 || d->nx < 3 || d->ny < 3)
        return set_error(LBM_ERR_INVALID, "channel2d needs a D2Q9 descriptor with nx, ny >= 3 and a mask");
    if (config_mode < 0 || config_mode > 2) return set_error(LBM_ERR_INVALID, "config_mode must be 0, 1 or 2");
    const int64_t nx = d->nx, ny = d->ny;
    // classes: 0 fluid, 1 solid, 2 inlet, 3 outlet, 4 solid cell on the inlet/outlet column
    for (int64_t y = 0; y < ny; ++y)
        for (int64_t x = 0; x < nx; ++x) {
            const double dx = (double)x - ox, dy = (double)y - oy;
            // circle + rows y = 0, ny-1 (cpp/d2q9_bgk_channel_packed.cpp:37-39)
            const bool solid = (dx * dx + dy * dy <= r * r) || y == 0 || y == ny - 1;
            const bool end_col = x == 0 || x == nx - 1;
            uint8_t k;
            if (solid)
                k = (end_col && !config_mode) ? 4 : 1;
            else if (x == 0)
                k = 2;
            else if (x == nx - 1)
                k = 3;
            else
                k = 0;
            mask[x + nx * y] = k;
        }
    d->n_classes = 5;
    set_class(d, 0, 0, 1, 0, 0, 0);
    set_class(d, 1, kSolidFlags, 0, 0, 0, 0);
    if (!config_mode) {
        // UX(0,:) = u_max; UX/UY/DENSITY(ON) = 0; DENSITY(0,:) = DENSITY(end,:) = 1  (:64-69)
        set_class(d, 2, LBM_CELL_SET_UX | LBM_CELL_SET_RHO, 1, u_in, 0, 0);
        set_class(d, 3, LBM_CELL_SET_RHO, 1, 0, 0, 0);
        set_class(d, 4, kSolidFlags, 1, 0, 0, 0);
    } else if (config_mode == 2) {
        set_class(d, 2, LBM_CELL_ZOUHE_VEL_XM, 1, u_in, 0, 0);
        set_class(d, 3, LBM_CELL_ZOUHE_RHO_XP, 1, 0, 0, 0);
        set_class(d, 4, kSolidFlags, 0, 0, 0, 0);
    } else {
        set_class(d, 2, LBM_CELL_EQUILIBRIUM | LBM_CELL_SET_RHO | LBM_CELL_SET_UX | LBM_CELL_SET_UY | LBM_CELL_SET_UZ,
                  1, u_in, 0, 0);
        set_class(d, 3, LBM_CELL_ZEROGRAD_XP, 1, 0, 0, 0);
        set_class(d, 4, kSolidFlags, 0, 0, 0, 0);
    }
    d->mask = mask;
    return LBM_OK;
}

int lbm_setup_duct3d(lbm_desc* d, uint8_t* mask, double u_in, double ox, double oy, double oz, double r) {
    if (!d || !mask || d->lattice != LBM_D3Q27 || d->nx < 3 || d->ny < 3 || d->nz < 3)
        return set_error(LBM_ERR_INVALID, "duct3d needs a D3Q27 descriptor with extents >= 3 and a mask");
    const int64_t nx = d->nx, ny = d->ny, nz = d->nz;
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                const double dx = (double)x - ox, dy = (double)y - oy, dz = (double)z - oz;
                const bool solid = (dx * dx + dy * dy + dz * dz <= r * r) || y == 0 || y == ny - 1 || z == 0 ||
                                   z == nz - 1;
                uint8_t k = solid ? 1 : (x == 0 ? 2 : (x == nx - 1 ? 3 : 0));
                mask[x + nx * (y + ny * z)] = k;
            }
    d->n_classes = 4;
    set_class(d, 0, 0, 1, 0, 0, 0);
    set_class(d, 1, kSolidFlags, 0, 0, 0, 0);
    set_class(d, 2, LBM_CELL_EQUILIBRIUM | LBM_CELL_SET_RHO | LBM_CELL_SET_UX | LBM_CELL_SET_UY | LBM_CELL_SET_UZ, 1,
              u_in, 0, 0);
    set_class(d, 3, LBM_CELL_ZEROGRAD_XP, 1, 0, 0, 0);
    d->mask = mask;
    return LBM_OK;
}

int lbm_mask_from_index_list(uint8_t* mask, int64_t n_cells, const int64_t* on, int64_t n_on, uint8_t cls) {
    if (!mask || n_cells < 0 || n_on < 0 || (n_on > 0 && !on)) return set_error(LBM_ERR_INVALID, "bad index list");
    if (cls >= LBM_MAX_CLASSES) return set_error(LBM_ERR_INVALID, "class id must be < 16");
    for (int64_t j = 0; j < n_on; ++j) {
        if (on[j] < 0 || on[j] >= n_cells) return set_error(LBM_ERR_INVALID, "index out of range in ON list");
        mask[on[j]] = cls;
    }
    return LBM_OK;
}

int lbm_mrt_collide_host(const lbm_desc* d, const double f_in[27], double rho, const double u[3], double f_out[27]) {
    if (!d || !f_in || !u || !f_out) return set_error(LBM_ERR_INVALID, "NULL argument");
    if (d->mrt_basis != LBM_MRT_REF && d->mrt_basis != LBM_MRT_GRAM_SCHMIDT)
        return set_error(LBM_ERR_INVALID, "unknown MRT basis");
    MrtCoef<double> k;
    mrt_coefficients(d->mrt_basis, d->mrt_s, k);
    double T[27];
    for (int i = 0; i < 27; ++i) T[D3Q27::slot(i)] = f_in[i];
    double q[11];
    q[0] = rho;
    q[1] = rho * u[0];
    q[2] = rho * u[1];
    q[3] = rho * u[2];
    q[4] = q[1] * u[0];
    q[5] = q[2] * u[1];
    q[6] = q[3] * u[2];
    q[7] = q[1] * u[1];
    q[8] = q[1] * u[2];
    q[9] = q[2] * u[2];
    q[10] = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    if (d->mrt_basis == LBM_MRT_REF) {
        mrt_forward<kMrtRef>(T);
        mrt_relax<kMrtRef>(T, q, k);
        mrt_inverse<kMrtRef>(T);
    } else {
        mrt_forward<kMrtGramSchmidt>(T);
        mrt_relax<kMrtGramSchmidt>(T, q, k);
        mrt_inverse<kMrtGramSchmidt>(T);
    }
    for (int i = 0; i < 27; ++i) f_out[i] = T[D3Q27::slot(i)];
    return LBM_OK;
}

}  // extern "C"
