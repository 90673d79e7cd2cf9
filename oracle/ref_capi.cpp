// C interface around the reference's own MDDriver (src/md_driver.cpp, thermostat.cpp,
// barostat.cpp compiled unchanged where they lie), so that tests can drive the real
// reference with ctypes. TEST INFRASTRUCTURE ONLY: this file is compiled by oracle/Makefile
// into oracle/_ref/libmdelast_ref.so and is used as a checker and as the timed CPU
// baseline, never by the product.
//
// Inputs follow the reference's md_driver_module constructor (md_driver_module.cpp:95-102):
// CGS units, node arrays exactly as get_potential.py hands them to TablePotential / EAM.
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "md_driver.hpp"

namespace {

struct RefHandle {
    std::vector<potential::PotentialPtr> pot;
    std::vector<potential::EAMPtr> eam;
    std::unique_ptr<MDDriver> d;
};

std::vector<double> vec(double const *p, long n) { return std::vector<double>(p, p + n); }

} // namespace

extern "C" {

// Pair tables: n_pot = n_types (n_types + 1) / 2 slots, each with n_r nodes (row k of the
// arrays is slot k). EAM: n_types functions with n_r (rho) and n_rho (F) nodes.
void *mref_create(int n_types, char const *interpolation, double rcut, double rmin_fatal,
                  double dr, int n_r, double const *phi, double const *dphi,
                  double const *d2phi, int has_eam, double eam_rcut, double rhomax_fatal,
                  double drho, int n_rho, double const *rho, double const *drho_dr,
                  double const *d2rho_dr2, double const *F, double const *dF,
                  double const *d2F, int n_atoms, double const *pos, double const *vel,
                  unsigned const *types, double const *mass, int ensemble, int coupling,
                  double T, int nchain, double const *q, double const *p_eta, double Nf_th,
                  double P, double w, double p_eps, double Tb, int nchain_b, double const *qb,
                  double const *p_eta_b, double Nf_b, double const *box9, int n_rg,
                  double const *rg, double Nf, double dt, int neighbors, double r_skin,
                  double fatal_conservation) {
    auto *h = new RefHandle();
    std::string const interp(interpolation);
    int const n_pot = n_types * (n_types + 1) / 2;
    for (int k = 0; k < n_pot; ++k) {
        long const o = static_cast<long>(k) * n_r;
        h->pot.push_back(std::make_shared<potential::TablePotential>(
            rcut, rmin_fatal, dr, vec(phi + o, n_r), vec(dphi + o, n_r), vec(d2phi + o, n_r),
            interp));
    }
    if (has_eam) {
        for (int t = 0; t < n_types; ++t) {
            long const orr = static_cast<long>(t) * n_r, orh = static_cast<long>(t) * n_rho;
            h->eam.push_back(std::make_shared<potential::EAM>(
                eam_rcut, rhomax_fatal, dr, drho, vec(rho + orr, n_r), vec(drho_dr + orr, n_r),
                vec(d2rho_dr2 + orr, n_r), vec(F + orh, n_rho), vec(dF + orh, n_rho),
                vec(d2F + orh, n_rho), interp));
        }
    }
    std::vector<Vector3d> P3, V3;
    for (int i = 0; i < n_atoms; ++i) {
        P3.emplace_back(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        V3.emplace_back(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
    Thermostat th(T, vec(q, nchain), vec(p_eta, nchain), Nf_th);
    Thermostat thb(Tb, vec(qb, nchain_b), vec(p_eta_b, nchain_b), Nf_b);
    Barostat baro(P, w, p_eps, thb);
    Eigen::Matrix3d hm;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            hm(r, c) = box9[3 * r + c];
    MDDriver::Box box(hm);
    std::vector<unsigned> ty(types, types + n_atoms);
    h->d = std::make_unique<MDDriver>(
        P3, V3, h->pot, h->eam, static_cast<MDDriver::Ensamble>(ensemble),
        static_cast<MDDriver::ThermostatCoupling>(coupling), th, baro, box, vec(rg, n_rg), Nf,
        vec(mass, n_types), ty, dt, neighbors != 0, r_skin, fatal_conservation);
    return h;
}

void mref_destroy(void *p) { delete static_cast<RefHandle *>(p); }

void mref_integrate(void *p, int n_steps) {
    auto *h = static_cast<RefHandle *>(p);
    for (int s = 0; s < n_steps; ++s)
        h->d->integrate();
}

void mref_calculate_neighbors(void *p) { static_cast<RefHandle *>(p)->d->calculate_neighbors(); }
void mref_calculate_forces(void *p) { static_cast<RefHandle *>(p)->d->calculate_forces(); }
void mref_set_sample_observables(void *p, int flag) {
    static_cast<RefHandle *>(p)->d->sample_observables = flag != 0;
}

// Scalar observables in a fixed order (the mdelast_observables layout of include/mdelast.h):
// 0 epot_eam_atom 1 epot_atom 2 ekin_atom 3 etot_atom 4 ekin_tot 5 etot_cons_initial
// 6 etot_cons 7 etot_cons_err 8 virial 9 total_laplacian 10 total_force2
// 11 temperature_kin 12 temperature_conf_inverse 13 pressure 14 time 15 cycle
// 16..21 born_stress_tensor 22..27 stress_tensor 28..63 born_elasticity_tensor (row major)
// 64..72 box h (row major) 73 barostat epsilon 74 barostat p_epsilon 75..77 momentum_tot
void mref_scalars(void *p, double *o) {
    MDDriver const &d = *static_cast<RefHandle *>(p)->d;
    o[0] = d.epot_eam_atom;
    o[1] = d.epot_atom;
    o[2] = d.ekin_atom;
    o[3] = d.etot_atom;
    o[4] = d.ekin_tot;
    o[5] = d.etot_cons_initial;
    o[6] = d.etot_cons;
    o[7] = d.etot_cons_err;
    o[8] = d.virial;
    o[9] = d.total_laplacian;
    o[10] = d.total_force2;
    o[11] = d.temperature_kin;
    o[12] = d.temperature_conf_inverse;
    o[13] = d.pressure;
    o[14] = d.time;
    o[15] = static_cast<double>(d.cycle);
    for (int i = 0; i < 6; ++i)
        o[16 + i] = d.born_stress_tensor(i);
    for (int i = 0; i < 6; ++i)
        o[22 + i] = d.stress_tensor(i);
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c)
            o[28 + 6 * r + c] = d.born_elasticity_tensor(r, c);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            o[64 + 3 * r + c] = d.box.h(r, c);
    o[73] = d.barostat.epsilon;
    o[74] = d.barostat.p_epsilon;
    o[75] = d.momentum_tot.x;
    o[76] = d.momentum_tot.y;
    o[77] = d.momentum_tot.z;
}

// Per-atom arrays: 0 positions 1 coordinates 2 velocities 3 forces (N x 3);
// 4 rho_eam 5 energies_pot 6 energies_kin 7 F_eam 8 dFdrho_eam 9 d2Fdrho2_eam (N)
void mref_atoms(void *p, int which, double *o) {
    MDDriver const &d = *static_cast<RefHandle *>(p)->d;
    unsigned const n = d.Nparticles;
    std::vector<Vector3d> const *v3 = nullptr;
    std::vector<double> const *v1 = nullptr;
    switch (which) {
    case 0: v3 = &d.positions; break;
    case 1: v3 = &d.coordinates; break;
    case 2: v3 = &d.velocities; break;
    case 3: v3 = &d.forces; break;
    case 4: v1 = &d.rho_eam; break;
    case 5: v1 = &d.energies_pot; break;
    case 6: v1 = &d.energies_kin; break;
    case 7: v1 = &d.F_eam; break;
    case 8: v1 = &d.dFdrho_eam; break;
    case 9: v1 = &d.d2Fdrho2_eam; break;
    default: return;
    }
    if (v3) {
        for (unsigned i = 0; i < n; ++i) {
            o[3 * i] = (*v3)[i].x;
            o[3 * i + 1] = (*v3)[i].y;
            o[3 * i + 2] = (*v3)[i].z;
        }
    } else {
        std::memcpy(o, v1->data(), sizeof(double) * n);
    }
}

// Thermostat chain state: which 0 = particle thermostat, 1 = barostat's thermostat.
int mref_chain(void *p, int which, double *p_eta, double *eta) {
    MDDriver const &d = *static_cast<RefHandle *>(p)->d;
    Thermostat const &t = which == 0 ? d.thermostat : d.barostat.thermostat;
    for (unsigned j = 0; j < t.nchain; ++j) {
        p_eta[j] = t.p_eta[j];
        eta[j] = t.eta[j];
    }
    return static_cast<int>(t.nchain);
}

// The half neighbour list of md_driver.cpp:279-298: point[N+1] and the first point[N]
// entries of neighbors. Returns point[N] (entries available), copying at most cap.
long mref_neighbors(void *p, int *point, int *neighbors, long cap) {
    MDDriver const &d = *static_cast<RefHandle *>(p)->d;
    if (d.point.empty())
        return -1;
    std::memcpy(point, d.point.data(), sizeof(int) * d.point.size());
    long const total = d.point[d.Nparticles];
    long const n = total < cap ? total : cap;
    std::memcpy(neighbors, d.neighbors.data(), sizeof(int) * static_cast<std::size_t>(n));
    return total;
}

// Pair correlation (md_driver.cpp:732-862): mode 0 total, 1 total + partial, 2 partial.
void mref_pair_correlation(void *p, int mode) {
    MDDriver &d = *static_cast<RefHandle *>(p)->d;
    if (mode == 0)
        d.calculate_pair_correlation();
    else if (mode == 1)
        d.calculate_pair_correlations();
    else
        d.calculate_partial_pair_correlation();
}

void mref_gr(void *p, double *gr, double *gr_partial) {
    MDDriver const &d = *static_cast<RefHandle *>(p)->d;
    std::memcpy(gr, d.gr.data(), sizeof(double) * d.gr.size());
    std::size_t k = 0;
    for (auto const &g : d.gr_partial) {
        std::memcpy(gr_partial + k, g.data(), sizeof(double) * g.size());
        k += g.size();
    }
}

// Table evaluation of pair slot k / EAM type t, for table-level checks:
// what 0 pair (V, dV, d2V) ; 1 rho (rho, drho, d2rho) ; 2 F (F, dF, d2F)
void mref_eval(void *p, int what, int k, double x, double *o3) {
    auto *h = static_cast<RefHandle *>(p);
    if (what == 0) {
        auto const v = h->pot[static_cast<std::size_t>(k)]->calculate(x);
        o3[0] = v.V;
        o3[1] = v.dVdr;
        o3[2] = v.d2Vdr2;
    } else if (what == 1) {
        auto &e = *h->eam[static_cast<std::size_t>(k)];
        o3[0] = e.rho(x);
        o3[1] = e.drhodr(x);
        o3[2] = e.d2rhodr2(x);
    } else {
        auto &e = *h->eam[static_cast<std::size_t>(k)];
        o3[0] = e.F(x);
        o3[1] = e.dFdrho(x);
        o3[2] = e.d2Fdrho2(x);
    }
}

} // extern "C"
