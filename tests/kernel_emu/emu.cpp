// Host build of the CUDA qp kernel source (plasticity_b200/csrc/cp_qp.cuh),
// used by the CPU test suite to check the device code path against the oracle
// without a GPU.  Exposes the oracle's entry-point signature: the history is
// taken in the oracle's qp-major layout and converted to the kernel's
// structure-of-arrays layout around the call.
#include <cstring>
#include <vector>

#include "../../include/cp_gpu.h"
#include "../../oracle/cp_oracle.h"
#include "../../plasticity_b200/csrc/cp_qp2.cuh"
#include "../../plasticity_b200/csrc/cp_qpref.cuh"

using namespace cp;

namespace {

LatDev make_lat(const cp_material_t& m) {
    LatDev hl;
    std::memset(&hl, 0, sizeof hl);
    hl.n = m.n_slip + m.n_twin;
    hl.ns = m.n_slip;
    hl.nw = m.n_twin;
    hl.twinning = m.twinning_enabled;
    std::memcpy(hl.C, m.elastic_stiffness, sizeof hl.C);
    std::memcpy(hl.m, m.slip_direction, sizeof hl.m);
    std::memcpy(hl.nn, m.slip_normal, sizeof hl.nn);
    std::memcpy(hl.q, m.latent_hardening, sizeof hl.q);
    std::memcpy(hl.s0, m.initial_slip_resistance, sizeof hl.s0);
    std::memcpy(hl.h0, m.initial_hardening_modulus, sizeof hl.h0);
    std::memcpy(hl.ss, m.saturation_stress, sizeof hl.ss);
    std::memcpy(hl.a, m.power_law_exponent, sizeof hl.a);
    std::memcpy(hl.C1, m.kinematic_c1, sizeof hl.C1);
    std::memcpy(hl.C2, m.kinematic_c2, sizeof hl.C2);
    hl.twin_thr = m.twin_threshold_fraction;
    hl.twin_sat = m.twin_saturation_factor;
    hl.twin_shear = m.twin_shear;
    return hl;
}

// AoS (qp-major, width w) <-> SoA (component-major)
void to_soa(const double* a, int64_t n, int w, double* s) {
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < w; ++c) s[c * n + i] = a[i * w + c];
}
void to_aos(const double* s, int64_t n, int w, double* a) {
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < w; ++c) a[i * w + c] = s[c * n + i];
}

int g_variant = 0;  // 0: qp_update2 (compact), 1: qp_update (plain), 2: ref::qp_update_ref

template <int NT, int PMAX>
void run_all(const LatDev& L, const Opts& o, const GroupDev& g, const double* F, int flag, double F_e, double F_r,
             double* P, double* T, double* dPdF, int32_t* stats, int32_t* status) {
    if (g_variant == 2) {
#pragma omp parallel
        {
            std::vector<double> w((size_t)ref::scratch_doubles(L.n));
#pragma omp for schedule(dynamic, 4)
            for (int64_t i = 0; i < g.count; ++i) {
                QpOut out;
                out.P = P ? P + 9 * i : nullptr;
                out.T = T ? T + 9 * i : nullptr;
                out.dPdF = (dPdF && flag == 1) ? dPdF + 81 * i : nullptr;
                out.scale = 1.0;
                const int st = ref::qp_update_ref(L, o, g, i, F + 9 * i, flag, F_e, F_r, out,
                                                  stats ? stats + 8 * i : nullptr, 0, w.data());
                if (status) status[i] = st;
            }
        }
        return;
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < g.count; ++i) {
        M3 Fk;
        for (int c = 0; c < 9; ++c) Fk.a[c] = F[9 * i + c];
        QpOut out;
        out.P = P ? P + 9 * i : nullptr;
        out.T = T ? T + 9 * i : nullptr;
        out.dPdF = (dPdF && flag == 1) ? dPdF + 81 * i : nullptr;
        out.scale = 1.0;
        double d2[21];  // the kernel keeps this slot in shared memory
        const int st = g_variant == 0
                           ? qp_update2<PMAX>(L, o, g, i, Fk, flag, F_e, F_r, out, stats ? stats + 8 * i : nullptr, 0,
                                              d2, 1)
                           : qp_update<NT, PMAX>(L, o, g, i, Fk, flag, F_e, F_r, out, stats ? stats + 8 * i : nullptr, 0);
        if (status) status[i] = st;
    }
}

}  // namespace

extern "C" void emu_set_variant(int v) { g_variant = v; }
extern "C" double emu_ref_pow(double x, double y) { return ref::ref_pow(x, y); }

extern "C" int emu_update(const cp_material_t* mat, const cp_options_t* opt, const or_state* st, const double* F,
                          int32_t flag, double F_e, double F_r, double* P, double* T, double* dPdF, int32_t* stats,
                          int32_t* status, int32_t nthreads) {
    (void)nthreads;
    const LatDev L = make_lat(*mat);
    const int64_t n = st->n_qp;
    const int nT = L.n, ns = L.ns, nw = L.nw;
    Opts o{opt->stress_tolerance, opt->max_slip_search_iterations, opt->max_solver_iterations,
           opt->enable_multiphase};
    std::vector<int64_t> qp(n);
    for (int64_t i = 0; i < n; ++i) qp[i] = i;
    struct F_ {
        double* aos;
        int w;
        std::vector<double> soa;
    };
    F_ fields[16] = {{st->Fp_conv, 9, {}},     {st->Fe_conv, 9, {}},       {st->s_conv, nT, {}},
                     {st->W_conv, nT, {}},     {st->rot_conv, 3, {}},      {st->rotnew_conv, 3, {}},
                     {st->twinfrac_conv, nw, {}}, {st->slipfrac_conv, ns, {}}, {st->Fp_iter, 9, {}},
                     {st->Fe_iter, 9, {}},     {st->s_iter, nT, {}},       {st->W_iter, nT, {}},
                     {st->rot_iter, 3, {}},    {st->rotnew_iter, 3, {}},   {st->twinfrac_iter, nw, {}},
                     {st->slipfrac_iter, ns, {}}};
    for (auto& f : fields) {
        f.soa.resize((size_t)n * f.w);
        to_soa(f.aos, n, f.w, f.soa.data());
    }
    std::vector<int> twin_c(st->twin_conv, st->twin_conv + n), twin_i(st->twin_iter, st->twin_iter + n);
    GroupDev g;
    g.count = n;
    g.qp = qp.data();
    double** slots[16] = {&g.Fp_c, &g.Fe_c, &g.s_c, &g.W_c, &g.rot_c, &g.rotnew_c, &g.tw_c, &g.sl_c,
                          &g.Fp_i, &g.Fe_i, &g.s_i, &g.W_i, &g.rot_i, &g.rotnew_i, &g.tw_i, &g.sl_i};
    for (int k = 0; k < 16; ++k) *slots[k] = fields[k].soa.data();
    g.twin_c = twin_c.data();
    g.twin_i = twin_i.data();
    g.where = nullptr;
    if (nT <= 16)
        run_all<16, 16>(L, o, g, F, flag, F_e, F_r, P, T, dPdF, stats, status);
    else if (nT <= 32)
        run_all<32, 32>(L, o, g, F, flag, F_e, F_r, P, T, dPdF, stats, status);
    else
        run_all<64, 64>(L, o, g, F, flag, F_e, F_r, P, T, dPdF, stats, status);
    for (int k = 8; k < 16; ++k) to_aos(fields[k].soa.data(), n, fields[k].w, fields[k].aos);
    for (int64_t i = 0; i < n; ++i) st->twin_iter[i] = twin_i[i];
    return 0;
}

// The batched solve of the compact update (lu_solve_b, one or two
// elimination steps per pass) against the plain one (lu_solve) on the same matrix: m x m with
// row stride ld, nrhs 1 or 9.  Returns 1 when solutions, factors (upper
// triangle), singular flags and pivot-ratio estimates are bit-identical; the
// only latitude is the sign of an exact zero (the plain form skips rows whose
// multiplier is zero, the batched one subtracts 0 * x) and NaN payloads.
static bool same_bits(double a, double b) {
    if (std::memcmp(&a, &b, sizeof a) == 0) return true;
    return (a == 0.0 && b == 0.0) || (a != a && b != b);
}
extern "C" int emu_lu_compare(const double* A0, const double* B0, int m, int ld, int nrhs, int pair) {
    std::vector<double> a1(A0, A0 + (size_t)m * ld), a2 = a1;
    std::vector<double> b1(B0, B0 + (size_t)m * nrhs), b2 = b1;
    double c1 = 0.0, c2 = 0.0;
    const int s1 = lu_solve(a1.data(), m, ld, b1.data(), nrhs, nrhs, &c1);
    int s2;
    if (pair)
        s2 = nrhs == 9 ? lu_solve_b<9, true>(a2.data(), m, ld, b2.data(), &c2)
                       : lu_solve_b<1, true>(a2.data(), m, ld, b2.data(), &c2);
    else
        s2 = nrhs == 9 ? lu_solve_b<9, false>(a2.data(), m, ld, b2.data(), &c2)
                       : lu_solve_b<1, false>(a2.data(), m, ld, b2.data(), &c2);
    if (s1 != s2 || !same_bits(c1, c2)) return 0;
    for (size_t k = 0; k < b1.size(); ++k)
        if (!same_bits(b1[k], b2[k])) return 0;
    for (int i = 0; i < m; ++i)
        for (int c = i; c < m; ++c)
            if (!same_bits(a1[(size_t)i * ld + c], a2[(size_t)i * ld + c])) return 0;
    return 1;
}
