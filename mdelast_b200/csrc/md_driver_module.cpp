// pybind11 module "md_driver_module" over the C-ABI of libmdelast_cuda.so.
//
// It exposes the classes, constructors, attributes and methods of mdelast's own binding
// (src/md_driver_module.cpp:16-224) under the same names, so that the reference's
// molecular_dynamics.py, get_potential.py and scripts run against it unchanged; a script
// picks the implementation by sys.path order. Everything the MD step computes comes from
// the GPU through include/mdelast.h; this file only converts arguments and results.
//
// Additions that the reference does not have are keyword-only: MDDriver(...,
// precision="fp64"|"mixed", device=0), and the module functions device_available() and
// set_default_precision().
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>
#include <pybind11/stl_bind.h>

#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "mdelast.h"

namespace py = pybind11;

namespace {

constexpr double kAngstrom = 1e-8;

void check(int rc) {
    if (rc == MDELAST_OK)
        return;
    std::string const msg = mdelast_last_error();
    if (rc == MDELAST_ERR_UNSUPPORTED)
        throw py::value_error(msg); // replaced below by NotImplementedError
    throw std::runtime_error(msg.empty() ? "mdelast error " + std::to_string(rc) : msg);
}

void check_ni(int rc) {
    if (rc == MDELAST_ERR_UNSUPPORTED) {
        PyErr_SetString(PyExc_NotImplementedError, mdelast_last_error());
        throw py::error_already_set();
    }
    check(rc);
}

// Every record of the sample ring of replica r (r < 0: a single driver), as arrays named
// like the attributes molecular_dynamics.py:1218-1238 appends per sampled step.
py::dict drain_dict(mdelast_driver *d, int r) {
    std::vector<mdelast_sample> all, buf(4096);
    int64_t lost_total = 0;
    for (;;) {
        int64_t n = 0, lost = 0;
        int64_t const cap = static_cast<int64_t>(buf.size());
        check(r < 0 ? mdelast_driver_drain_samples(d, buf.data(), cap, &n, &lost)
                    : mdelast_batch_drain_samples(d, r, buf.data(), cap, &n, &lost));
        lost_total += lost;
        all.insert(all.end(), buf.begin(), buf.begin() + n);
        if (n < cap)
            break;
    }
    size_t const n = all.size();
    py::dict out;
    auto col = [&](char const *name, double mdelast_sample::*f) {
        py::array_t<double> a(n);
        for (size_t i = 0; i < n; ++i)
            a.mutable_data()[i] = all[i].*f;
        out[name] = a;
    };
    col("time", &mdelast_sample::time);
    col("cycle", &mdelast_sample::cycle);
    col("temperature_kin", &mdelast_sample::temperature_kin);
    col("temperature_conf_inverse", &mdelast_sample::temperature_conf_inverse);
    col("total_laplacian", &mdelast_sample::total_laplacian);
    col("total_force2", &mdelast_sample::total_force2);
    col("pressure", &mdelast_sample::pressure);
    col("etot_atom", &mdelast_sample::etot_atom);
    col("epot_atom", &mdelast_sample::epot_atom);
    col("epot_eam_atom", &mdelast_sample::epot_eam_atom);
    col("ekin_atom", &mdelast_sample::ekin_atom);
    col("etot_cons", &mdelast_sample::etot_cons);
    col("etot_cons_err", &mdelast_sample::etot_cons_err);
    col("volume", &mdelast_sample::volume);
    py::array_t<double> st({n, size_t(6)}), bs({n, size_t(6)}), be({n, size_t(6), size_t(6)});
    py::array_t<uint32_t> status(n);
    for (size_t i = 0; i < n; ++i) {
        for (int k = 0; k < 6; ++k) {
            st.mutable_data()[6 * i + k] = all[i].stress_tensor[k];
            bs.mutable_data()[6 * i + k] = all[i].born_stress_tensor[k];
        }
        int q = 0;
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b)
                be.mutable_data()[36 * i + 6 * a + b] =
                    b >= a ? all[i].born_elasticity_tensor[q++] : 0.;
        status.mutable_data()[i] = static_cast<uint32_t>(all[i].status);
    }
    out["stress_tensor"] = st;
    out["born_stress_tensor"] = bs;
    out["born_elasticity_tensor"] = be;
    out["status"] = status;
    out["lost"] = lost_total;
    return out;
}

py::dict fluct_dict(mdelast_fluct const &f) {
    py::dict out;
    out["n"] = f.n;
    out["n_atoms"] = f.n_atoms;
    py::array_t<double> mean(9), M({size_t(9), size_t(9)}), cb({size_t(6), size_t(6)});
    std::copy(f.mean, f.mean + 9, mean.mutable_data());
    int q = 0;
    for (int a = 0; a < 9; ++a)
        for (int b = a; b < 9; ++b, ++q)
            M.mutable_data()[9 * a + b] = M.mutable_data()[9 * b + a] = f.comoment[q];
    q = 0;
    for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b)
            cb.mutable_data()[6 * a + b] = b >= a ? f.born_el_mean[q++] : 0.;
    out["mean"] = mean;
    out["comoment"] = M;
    out["born_el_mean"] = cb;
    return out;
}

py::dict elastic_dict(mdelast_fluct const &f, int ensemble, double T, double P) {
    py::array_t<double> C({size_t(6), size_t(6)});
    double sm[6];
    check(mdelast_elastic_constants(&f, ensemble, T, P, C.mutable_data(), sm));
    py::dict out;
    out["C"] = C;
    out["C11"] = sm[0];
    out["C12"] = sm[1];
    out["C44"] = sm[2];
    out["bulk_modulus"] = sm[3];
    out["compressibility"] = sm[4];
    out["volume_thermal_expansion"] = sm[5];
    out["n_samples"] = f.n;
    return out;
}

py::dict autotune_dict(mdelast_driver *d, int n_repeat, int steps_rebuild = -1) {
    int32_t c[4];
    double ms[2];
    if (steps_rebuild >= 0)
        check(mdelast_driver_autotune_steps(d, n_repeat, steps_rebuild, c, ms));
    else
        check(mdelast_driver_autotune(d, n_repeat, c, ms));
    py::dict out;
    out["tpa_density"] = c[0];
    out["tpa_force"] = c[1];
    out["blocks_density"] = c[2];
    out["blocks_force"] = c[3];
    out["ms_density"] = ms[0];
    out["ms_force"] = ms[1];
    int32_t on = 0;
    check(mdelast_driver_get_force_staging(d, &on, nullptr));
    out["force_staged"] = on != 0;
    return out;
}

// the force-pass variant with the tables staged in shared memory (read / switch)
py::object force_staging_get(mdelast_driver *d) {
    int32_t on = 0, avail = 0;
    check(mdelast_driver_get_force_staging(d, &on, &avail));
    if (!avail)
        return py::none();
    return py::bool_(on != 0);
}

int parse_interp(std::string const &name) {
    if (name == "quintic")
        return MDELAST_QUINTIC;
    if (name == "bspline")
        return MDELAST_BSPLINE;
    throw py::value_error("FATAL: unknown table interpolation '" + name +
                          "' (use 'quintic' or 'bspline')");
}

std::string default_precision = "fp64";

// vector3d.hpp:5-107 (the parts the binding exposes)
struct Vector3d {
    double x = 0, y = 0, z = 0;
    Vector3d() = default;
    Vector3d(double x_, double y_, double z_) : x(x_), y(y_), z(z_) {}
    double length2() const { return x * x + y * y + z * z; }
    double length() const { return std::sqrt(length2()); }
};

struct PotentialValue {
    double V, dVdr, d2Vdr2;
};

struct PairHandle {
    mdelast_pair *p = nullptr;
    ~PairHandle() { mdelast_pair_destroy(p); }
};
struct EamHandle {
    mdelast_eam *e = nullptr;
    ~EamHandle() { mdelast_eam_destroy(e); }
};

class Potential {
  public:
    explicit Potential(std::shared_ptr<PairHandle> h) : h_(std::move(h)) {
        check(mdelast_pair_info(h_->p, &rcut, nullptr, nullptr));
    }
    virtual ~Potential() = default;
    PotentialValue calculate(double r) const {
        double o[3];
        check(mdelast_pair_eval(h_->p, r, o));
        return {o[0], o[1], o[2]};
    }
    mdelast_pair const *handle() const { return h_->p; }
    double rcut = 0;

  private:
    std::shared_ptr<PairHandle> h_;
};

std::shared_ptr<PairHandle> make_pair_handle(int rc, mdelast_pair *p) {
    check_ni(rc);
    auto h = std::make_shared<PairHandle>();
    h->p = p;
    return h;
}

class Morse : public Potential {
  public:
    Morse(double rcut_, double D_, double alpha_, double r0_)
        : Potential(create(rcut_, D_, alpha_, r0_)), D(D_), alpha(alpha_), r0(r0_) {}
    double D, alpha, r0;

  private:
    static std::shared_ptr<PairHandle> create(double rc, double D, double a, double r0) {
        mdelast_pair *p = nullptr;
        int const rcode = mdelast_pair_morse_create(rc, D, a, r0, &p);
        return make_pair_handle(rcode, p);
    }
};

class LennardJones : public Potential {
  public:
    LennardJones(double rcut_, double epsilon_, double sigma_)
        : Potential(create(rcut_, epsilon_, sigma_)), epsilon(epsilon_), sigma(sigma_) {}
    double epsilon, sigma;

  private:
    static std::shared_ptr<PairHandle> create(double rc, double e, double s) {
        mdelast_pair *p = nullptr;
        int const rcode = mdelast_pair_lj_create(rc, e, s, &p);
        return make_pair_handle(rcode, p);
    }
};

class TablePotential : public Potential {
  public:
    TablePotential(double rcut_, double rmin_fatal_, double dr, std::vector<double> const &v,
                   std::vector<double> const &dv, std::vector<double> const &d2v,
                   std::string const &interpolation_ = "quintic")
        : Potential(create(rcut_, rmin_fatal_, dr, v, dv, d2v, interpolation_)),
          rmin_fatal(rmin_fatal_), interpolation(interpolation_) {}
    double rmin_fatal;
    std::string interpolation;

  private:
    static std::shared_ptr<PairHandle> create(double rc, double rmin, double dr,
                                              std::vector<double> const &v,
                                              std::vector<double> const &dv,
                                              std::vector<double> const &d2v,
                                              std::string const &interp) {
        int const code = parse_interp(interp);
        if (dv.size() != v.size() || d2v.size() != v.size())
            throw py::value_error("FATAL: QuinticTable needs equal array sizes");
        mdelast_pair *p = nullptr;
        int const rcode = mdelast_pair_table_create(rc, rmin, dr, static_cast<int64_t>(v.size()),
                                                    v.data(), dv.data(), d2v.data(), code, &p);
        return make_pair_handle(rcode, p);
    }
};

class EAM {
  public:
    EAM(double rcut_, double rhomax_fatal_, double dr, double drho, std::vector<double> const &rho_,
        std::vector<double> const &drho_, std::vector<double> const &d2rho_,
        std::vector<double> const &F_, std::vector<double> const &dF_,
        std::vector<double> const &d2F_, std::string const &interpolation_ = "quintic")
        : rcut(rcut_), rhomax_fatal(rhomax_fatal_), interpolation(interpolation_) {
        int const code = parse_interp(interpolation_);
        if (drho_.size() != rho_.size() || d2rho_.size() != rho_.size() ||
            dF_.size() != F_.size() || d2F_.size() != F_.size())
            throw py::value_error("FATAL: QuinticTable needs equal array sizes");
        mdelast_eam *e = nullptr;
        check_ni(mdelast_eam_create(rcut_, rhomax_fatal_, dr, drho,
                                    static_cast<int64_t>(rho_.size()), rho_.data(), drho_.data(),
                                    d2rho_.data(), static_cast<int64_t>(F_.size()), F_.data(),
                                    dF_.data(), d2F_.data(), code, &e));
        h_ = std::make_shared<EamHandle>();
        h_->e = e;
    }
    double eval(int what, double x) const {
        double v;
        check(mdelast_eam_eval(h_->e, what, x, &v));
        return v;
    }
    mdelast_eam const *handle() const { return h_->e; }
    double rcut, rhomax_fatal;
    std::string interpolation;

  private:
    std::shared_ptr<EamHandle> h_;
};

using PotentialPtr = std::shared_ptr<Potential>;
using EAMPtr = std::shared_ptr<EAM>;

// md_driver.hpp:28-37
struct Box {
    explicit Box(py::array_t<double, py::array::c_style | py::array::forcecast> h_) {
        if (h_.ndim() != 2 || h_.shape(0) != 3 || h_.shape(1) != 3)
            throw py::value_error("Box needs a 3x3 matrix");
        auto r = h_.unchecked<2>();
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                h[3 * a + b] = r(a, b);
    }
    Box() = default;
    double h[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double volume() const {
        return h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) +
               h[2] * (h[3] * h[7] - h[4] * h[6]);
    }
    double length() const { return (h[0] + h[4] + h[8]) / 3.; }
    py::array_t<double> h_array() const {
        py::array_t<double> a({3, 3});
        auto w = a.mutable_unchecked<2>();
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                w(r, c) = h[3 * r + c];
        return a;
    }
};

// thermostat.hpp:9-38 / barostat.hpp:6-17 (state holders)
struct Thermostat {
    Thermostat(double T, std::vector<double> q_, std::vector<double> p_eta_, double Nf_)
        : temperature(T), q(std::move(q_)), p_eta(std::move(p_eta_)),
          eta(p_eta.size(), 0.), nchain(static_cast<unsigned>(p_eta.size())), Nf(Nf_) {
        if (!(T > 0.) || q.size() != p_eta.size() || p_eta.empty() || !(Nf > 0.))
            throw py::value_error("Thermostat needs T > 0, Nf > 0 and equal non-empty q, p_eta");
    }
    double temperature;
    std::vector<double> q, p_eta, eta;
    unsigned nchain;
    double Nf;
};

struct Barostat {
    Barostat(double P, double w_, double p_eps, Thermostat const &t)
        : pressure(P), w(w_), epsilon(0.), p_epsilon(p_eps), thermostat(t) {
        if (!(w_ > 0.))
            throw py::value_error("Barostat needs w > 0");
    }
    double pressure, w, epsilon, p_epsilon;
    Thermostat thermostat;
};

struct BarostatFlex {
    BarostatFlex(double P, double w_, py::array_t<double> pg_, Thermostat const &t)
        : pressure(P), w(w_), pg(pg_), thermostat(t) {}
    double pressure, w;
    py::array_t<double> pg;
    Thermostat thermostat;
};

enum Ensamble { NVE = MDELAST_NVE, NVT = MDELAST_NVT, NPT = MDELAST_NPT, NPT_FLEX = MDELAST_NPT_FLEX };
enum ThermostatCoupling {
    THERMOSTAT_KINETIC = MDELAST_THERMOSTAT_KINETIC,
    THERMOSTAT_CONFIGURATIONAL = MDELAST_THERMOSTAT_CONFIGURATIONAL,
    THERMOSTAT_AVERAGE = MDELAST_THERMOSTAT_AVERAGE
};

class MDDriver {
  public:
    MDDriver(std::vector<Vector3d> const &positions, std::vector<Vector3d> const &velocities,
             std::vector<PotentialPtr> const &pot, std::vector<EAMPtr> const &eam,
             Ensamble ensamble_, ThermostatCoupling coupling, Thermostat const &thermostat,
             Barostat const &barostat, Box const &box, std::vector<double> const &rg_,
             double Nf, std::vector<double> const &mass_, std::vector<unsigned> const &types_,
             double dt, bool neighbors, double r_skin, double fatal_conservation_,
             std::string const &precision, int device)
        : ensamble(ensamble_), thermostat_coupling(coupling), box_initial(box), rg(rg_),
          dt_global(dt), fatal_conservation(fatal_conservation_), mass(mass_), types(types_),
          pot_(pot), eam_(eam), thermo_T_(thermostat.temperature), thermo_Nf_(thermostat.Nf),
          baro_P_(barostat.pressure), baro_w_(barostat.w),
          baro_thermo_T_(barostat.thermostat.temperature), baro_Nf_(barostat.thermostat.Nf) {
        size_t const N = positions.size();
        if (velocities.size() != N || types.size() != N)
            throw py::value_error("positions, velocities and types differ in length");
        std::vector<double> pos(3 * N), vel(3 * N);
        for (size_t i = 0; i < N; ++i) {
            pos[3 * i] = positions[i].x;
            pos[3 * i + 1] = positions[i].y;
            pos[3 * i + 2] = positions[i].z;
            vel[3 * i] = velocities[i].x;
            vel[3 * i + 1] = velocities[i].y;
            vel[3 * i + 2] = velocities[i].z;
        }
        std::vector<mdelast_pair const *> ph;
        for (auto const &p : pot)
            ph.push_back(p ? p->handle() : nullptr);
        std::vector<mdelast_eam const *> eh;
        for (auto const &e : eam)
            eh.push_back(e ? e->handle() : nullptr);
        size_t const nt = mass.size();
        if (ph.size() != nt * (nt + 1) / 2)
            throw py::value_error("PotentialVector needs n_types (n_types + 1) / 2 entries");
        gr.assign(rg.size(), 0.); // md_driver.cpp:39-40
        gr_partial.assign(nt * (nt + 1) / 2, std::vector<double>(rg.size(), 0.));
        Nparticles_per_type.assign(nt, 0);
        for (unsigned t : types)
            if (t < nt)
                Nparticles_per_type[t] += 1;
        std::string prec = precision.empty() ? default_precision : precision;
        mdelast_driver_config c{};
        c.n_atoms = static_cast<int32_t>(N);
        c.n_types = static_cast<int32_t>(nt);
        c.positions = pos.data();
        c.velocities = vel.data();
        c.types = reinterpret_cast<uint32_t const *>(types.data());
        c.mass = mass.data();
        c.pair = ph.data();
        c.eam = eh.data();
        c.n_eam = static_cast<int32_t>(eh.size());
        c.ensemble = ensamble;
        c.coupling = coupling;
        c.thermo_T = thermostat.temperature;
        c.thermo_nchain = static_cast<int32_t>(thermostat.nchain);
        c.thermo_q = thermostat.q.data();
        c.thermo_p_eta = thermostat.p_eta.data();
        c.thermo_Nf = thermostat.Nf;
        c.baro_P = barostat.pressure;
        c.baro_w = barostat.w;
        c.baro_p_eps = barostat.p_epsilon;
        c.baro_thermo_T = barostat.thermostat.temperature;
        c.baro_nchain = static_cast<int32_t>(barostat.thermostat.nchain);
        c.baro_q = barostat.thermostat.q.data();
        c.baro_p_eta = barostat.thermostat.p_eta.data();
        c.baro_Nf = barostat.thermostat.Nf;
        for (int k = 0; k < 9; ++k)
            c.box[k] = box.h[k];
        c.n_rg = static_cast<int32_t>(rg.size());
        c.rg = rg.data();
        c.Nf = Nf;
        c.dt = dt;
        c.neighbors = neighbors ? 1 : 0;
        c.r_skin = r_skin;
        c.fatal_conservation = fatal_conservation;
        c.precision = prec == "mixed" ? MDELAST_PRECISION_MIXED : MDELAST_PRECISION_FP64;
        if (prec != "mixed" && prec != "fp64")
            throw py::value_error("precision must be 'fp64' or 'mixed'");
        c.device = device;
        thermo_q_ = thermostat.q;
        baro_q_ = barostat.thermostat.q;
        mdelast_driver *d = nullptr;
        check_ni(mdelast_driver_create(&c, &d));
        d_ = d;
        precision_ = prec;
    }
    ~MDDriver() { mdelast_driver_destroy(d_); }
    MDDriver(MDDriver const &) = delete;
    MDDriver &operator=(MDDriver const &) = delete;

    mdelast_observables const &obs() {
        check(mdelast_driver_get_observables(d_, &obs_));
        return obs_;
    }
    void integrate() { check(mdelast_driver_integrate(d_, 1)); }
    void integrate_n(int n) { check(mdelast_driver_integrate(d_, n)); }
    void calculate_neighbors() { check_ni(mdelast_driver_calculate_neighbors(d_)); }
    bool get_sample() const {
        int32_t f = 0;
        check(mdelast_driver_get_sample_observables(d_, &f));
        return f != 0;
    }
    void set_sample(bool f) { check(mdelast_driver_set_sample_observables(d_, f ? 1 : 0)); }

    std::vector<double> atoms1(int field) {
        std::vector<double> v(types.size());
        check(mdelast_driver_get_atoms(d_, field, v.data()));
        return v;
    }
    std::vector<Vector3d> atoms3(int field) {
        size_t const N = types.size();
        std::vector<double> v(3 * N);
        check(mdelast_driver_get_atoms(d_, field, v.data()));
        std::vector<Vector3d> out(N);
        for (size_t i = 0; i < N; ++i)
            out[i] = Vector3d(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        return out;
    }
    py::array_t<double> atoms_array(int field) {
        size_t const N = types.size();
        bool const three = field <= MDELAST_ATOM_FORCES;
        py::array_t<double> a = three ? py::array_t<double>({N, size_t(3)}) : py::array_t<double>(N);
        check(mdelast_driver_get_atoms(d_, field, a.mutable_data()));
        return a;
    }
    Thermostat thermostat() {
        std::vector<double> p(thermo_q_.size()), e(thermo_q_.size());
        int32_t n = 0;
        check(mdelast_driver_get_chain(d_, 0, nullptr, p.data(), e.data(), &n));
        Thermostat t(thermo_T_, thermo_q_, p, thermo_Nf_);
        t.eta = e;
        return t;
    }
    Barostat barostat() {
        std::vector<double> p(baro_q_.size()), e(baro_q_.size());
        int32_t n = 0;
        check(mdelast_driver_get_chain(d_, 1, nullptr, p.data(), e.data(), &n));
        Thermostat t(baro_thermo_T_, baro_q_, p, baro_Nf_);
        t.eta = e;
        mdelast_observables const &o = obs();
        Barostat b(baro_P_, baro_w_, o.baro_p_epsilon, t);
        b.epsilon = o.baro_epsilon;
        return b;
    }
    Box box() {
        mdelast_observables const &o = obs();
        Box b;
        for (int k = 0; k < 9; ++k)
            b.h[k] = o.box[k];
        return b;
    }
    py::tuple neighbor_list() {
        size_t const N = types.size();
        py::array_t<int32_t> point(N + 1);
        int64_t total = 0;
        check_ni(mdelast_driver_get_neighbors(d_, point.mutable_data(), nullptr, 0, &total));
        py::array_t<int32_t> nb(static_cast<size_t>(total));
        check(mdelast_driver_get_neighbors(d_, point.mutable_data(), nb.mutable_data(), total,
                                           &total));
        return py::make_tuple(point, nb);
    }
    void pair_correlation(int mode) {
        check_ni(mdelast_driver_pair_correlation(d_, mode));
        size_t const nt = mass.size(), np = nt * (nt + 1) / 2, ng = rg.size();
        std::vector<double> g(ng), gp(np * ng);
        check(mdelast_driver_get_gr(d_, g.data(), gp.data()));
        if (mode != 2)
            gr = g;
        if (mode != 0) {
            gr_partial.assign(np, std::vector<double>(ng));
            for (size_t k = 0; k < np; ++k)
                for (size_t q = 0; q < ng; ++q)
                    gr_partial[k][q] = gp[k * ng + q];
        }
    }
    void synchronize() { check(mdelast_driver_synchronize(d_)); }
    void set_sample_ring(int capacity) { check(mdelast_driver_set_sample_ring(d_, capacity)); }
    py::dict autotune(int n_repeat) { return autotune_dict(d_, n_repeat); }
    py::dict autotune_steps(int n, int rebuild_every) {
        return autotune_dict(d_, n, rebuild_every);
    }
    py::object force_staging() { return force_staging_get(d_); }
    py::tuple list_capacity() {
        int32_t m = 0, g = 0;
        check(mdelast_driver_list_capacity(d_, &m, &g));
        return py::make_tuple(m, g);
    }
    void set_force_staging(bool on) { check(mdelast_driver_set_force_staging(d_, on ? 1 : 0)); }
    void set_launch(int td, int tf, int bd, int bf) {
        check(mdelast_driver_set_launch(d_, td, tf, bd, bf));
    }
    void set_pair_list(double f) { check(mdelast_driver_set_pair_list(d_, f)); }
    py::dict drain_samples() { return drain_dict(d_, -1); }
    void fluctuation_start() { check(mdelast_driver_fluct_start(d_)); }
    mdelast_fluct fluct() {
        mdelast_fluct f;
        check(mdelast_driver_get_fluct(d_, &f));
        return f;
    }
    py::dict fluctuations() { return fluct_dict(fluct()); }
    py::dict elastic_constants(py::object T, py::object P) {
        return elastic_dict(fluct(), static_cast<int>(ensamble),
                            T.is_none() ? thermo_T_ : T.cast<double>(),
                            P.is_none() ? baro_P_ : P.cast<double>());
    }
    double run(int n, int rebuild_every, int sample_every, bool timed) {
        float ms = 0.f;
        check(mdelast_driver_run(d_, n, rebuild_every, sample_every, timed ? &ms : nullptr));
        return ms;
    }
    std::vector<double> kernel_times(int n) {
        std::vector<double> t(MDELAST_N_KERNEL_TIMES);
        check(mdelast_driver_kernel_times(d_, n, t.data()));
        return t;
    }

    Ensamble ensamble;
    ThermostatCoupling thermostat_coupling;
    Box box_initial;
    std::vector<double> rg, gr, mass_dummy;
    std::vector<std::vector<double>> gr_partial;
    double dt_global, fatal_conservation;
    std::vector<double> mass;
    std::vector<unsigned> types;
    std::vector<unsigned> Nparticles_per_type;
    std::string precision_;

  private:
    mdelast_driver *d_ = nullptr;
    mdelast_observables obs_{};
    std::vector<PotentialPtr> pot_;
    std::vector<EAMPtr> eam_;
    double thermo_T_, thermo_Nf_, baro_P_, baro_w_, baro_thermo_T_, baro_Nf_;
    std::vector<double> thermo_q_, baro_q_;
};

py::array_t<double> vec6(double const *v) {
    py::array_t<double> a(6);
    std::copy(v, v + 6, a.mutable_data());
    return a;
}

py::dict obs_dict(mdelast_observables const &o) {
    py::dict d;
    d["epot_eam_atom"] = o.epot_eam_atom;
    d["epot_atom"] = o.epot_atom;
    d["ekin_atom"] = o.ekin_atom;
    d["etot_atom"] = o.etot_atom;
    d["etot_cons"] = o.etot_cons;
    d["etot_cons_err"] = o.etot_cons_err;
    d["virial"] = o.virial;
    d["total_laplacian"] = o.total_laplacian;
    d["total_force2"] = o.total_force2;
    d["temperature_kin"] = o.temperature_kin;
    d["temperature_conf_inverse"] = o.temperature_conf_inverse;
    d["pressure"] = o.pressure;
    d["time"] = o.time;
    d["cycle"] = static_cast<unsigned long long>(o.cycle);
    d["born_stress_tensor"] = vec6(o.born_stress_tensor);
    d["stress_tensor"] = vec6(o.stress_tensor);
    py::array_t<double> cb({6, 6});
    std::copy(o.born_elasticity_tensor, o.born_elasticity_tensor + 36, cb.mutable_data());
    d["born_elasticity_tensor"] = cb;
    d["volume"] = o.box[0] * (o.box[4] * o.box[8]);
    d["box"] = py::make_tuple(o.box[0], o.box[4], o.box[8]);
    d["baro_epsilon"] = o.baro_epsilon;
    d["baro_p_epsilon"] = o.baro_p_epsilon;
    d["status"] = o.status;
    return d;
}

// Every replica's observables in one dict of arrays with the replica as the first axis
// (the fields of obs_dict).
py::dict obs_dict_all(std::vector<mdelast_observables> const &o) {
    size_t const n = o.size();
    py::dict d;
    auto col = [&](char const *name, double mdelast_observables::*f) {
        py::array_t<double> a(n);
        for (size_t i = 0; i < n; ++i)
            a.mutable_data()[i] = o[i].*f;
        d[name] = a;
    };
    col("epot_eam_atom", &mdelast_observables::epot_eam_atom);
    col("epot_atom", &mdelast_observables::epot_atom);
    col("ekin_atom", &mdelast_observables::ekin_atom);
    col("etot_atom", &mdelast_observables::etot_atom);
    col("etot_cons", &mdelast_observables::etot_cons);
    col("etot_cons_err", &mdelast_observables::etot_cons_err);
    col("virial", &mdelast_observables::virial);
    col("total_laplacian", &mdelast_observables::total_laplacian);
    col("total_force2", &mdelast_observables::total_force2);
    col("temperature_kin", &mdelast_observables::temperature_kin);
    col("temperature_conf_inverse", &mdelast_observables::temperature_conf_inverse);
    col("pressure", &mdelast_observables::pressure);
    col("time", &mdelast_observables::time);
    col("baro_epsilon", &mdelast_observables::baro_epsilon);
    col("baro_p_epsilon", &mdelast_observables::baro_p_epsilon);
    py::array_t<unsigned long long> cyc(n);
    py::array_t<uint32_t> status(n);
    py::array_t<double> vol(n), bs({n, size_t(6)}), st({n, size_t(6)}), box({n, size_t(3)}),
        cb({n, size_t(6), size_t(6)});
    for (size_t i = 0; i < n; ++i) {
        cyc.mutable_data()[i] = static_cast<unsigned long long>(o[i].cycle);
        status.mutable_data()[i] = o[i].status;
        vol.mutable_data()[i] = o[i].box[0] * (o[i].box[4] * o[i].box[8]);
        for (int k = 0; k < 3; ++k)
            box.mutable_data()[3 * i + k] = o[i].box[4 * k];
        for (int k = 0; k < 6; ++k) {
            bs.mutable_data()[6 * i + k] = o[i].born_stress_tensor[k];
            st.mutable_data()[6 * i + k] = o[i].stress_tensor[k];
        }
        std::copy(o[i].born_elasticity_tensor, o[i].born_elasticity_tensor + 36,
                  cb.mutable_data() + 36 * i);
    }
    d["cycle"] = cyc;
    d["born_stress_tensor"] = bs;
    d["stress_tensor"] = st;
    d["born_elasticity_tensor"] = cb;
    d["volume"] = vol;
    d["box"] = box;
    d["status"] = status;
    return d;
}

// Many independent replicas sharing one potential, advanced together on one GPU (new in
// this implementation; the reference runs replicas as separate processes). Per replica:
// positions (N,3) and velocities (N,3) arrays [cgs], types, ensemble, thermostat and
// barostat, box edges, Nf; shared: potentials, masses, dt, list settings, precision.
class BatchedMDDriver {
  public:
    BatchedMDDriver(std::vector<py::array_t<double, py::array::c_style | py::array::forcecast>> const &positions,
                    std::vector<py::array_t<double, py::array::c_style | py::array::forcecast>> const &velocities,
                    std::vector<py::array_t<uint32_t, py::array::c_style | py::array::forcecast>> const &types,
                    std::vector<PotentialPtr> const &pot, std::vector<EAMPtr> const &eam,
                    std::vector<Ensamble> const &ensembles, std::vector<Thermostat> const &thermostats,
                    std::vector<Barostat> const &barostats, std::vector<Box> const &boxes,
                    std::vector<double> const &Nf, std::vector<double> const &mass, double dt,
                    bool neighbors, double r_skin, double fatal_conservation,
                    std::string const &precision, int device, std::vector<double> const &rg)
        : pot_(pot), eam_(eam), mass_(mass) {
        size_t const R = positions.size();
        if (R == 0 || velocities.size() != R || types.size() != R || ensembles.size() != R ||
            thermostats.size() != R || barostats.size() != R || boxes.size() != R ||
            Nf.size() != R)
            throw py::value_error("every per-replica list needs one entry per replica");
        std::vector<mdelast_pair const *> ph;
        for (auto const &p : pot)
            ph.push_back(p->handle());
        std::vector<mdelast_eam const *> eh;
        for (auto const &e : eam)
            eh.push_back(e->handle());
        std::vector<mdelast_driver_config> cfg(R);
        std::string const prec = precision.empty() ? default_precision : precision;
        for (size_t r = 0; r < R; ++r) {
            auto const &P = positions[r];
            auto const &V = velocities[r];
            size_t const N = static_cast<size_t>(types[r].size());
            if (P.size() != static_cast<py::ssize_t>(3 * N) || V.size() != static_cast<py::ssize_t>(3 * N))
                throw py::value_error("positions/velocities of a replica must be (N, 3)");
            mdelast_driver_config &c = cfg[r];
            c = mdelast_driver_config{};
            c.n_atoms = static_cast<int32_t>(N);
            c.n_types = static_cast<int32_t>(mass.size());
            c.positions = P.data();
            c.velocities = V.data();
            c.types = types[r].data();
            c.mass = mass_.data();
            c.pair = ph.data();
            c.eam = eh.data();
            c.n_eam = static_cast<int32_t>(eh.size());
            c.ensemble = ensembles[r];
            c.coupling = MDELAST_THERMOSTAT_KINETIC;
            Thermostat const &th = thermostats[r];
            Barostat const &b = barostats[r];
            c.thermo_T = th.temperature;
            c.thermo_nchain = static_cast<int32_t>(th.nchain);
            c.thermo_q = th.q.data();
            c.thermo_p_eta = th.p_eta.data();
            c.thermo_Nf = th.Nf;
            c.baro_P = b.pressure;
            c.baro_w = b.w;
            c.baro_p_eps = b.p_epsilon;
            c.baro_thermo_T = b.thermostat.temperature;
            c.baro_nchain = static_cast<int32_t>(b.thermostat.nchain);
            c.baro_q = b.thermostat.q.data();
            c.baro_p_eta = b.thermostat.p_eta.data();
            c.baro_Nf = b.thermostat.Nf;
            for (int k = 0; k < 9; ++k)
                c.box[k] = boxes[r].h[k];
            c.n_rg = static_cast<int32_t>(rg.size());
            c.rg = rg.data();
            c.Nf = Nf[r];
            c.dt = dt;
            c.neighbors = neighbors ? 1 : 0;
            c.r_skin = r_skin;
            c.fatal_conservation = fatal_conservation;
            c.precision = prec == "mixed" ? MDELAST_PRECISION_MIXED : MDELAST_PRECISION_FP64;
            c.device = device;
            counts_.push_back(N);
            ens_.push_back(c.ensemble);
            T_.push_back(th.temperature);
            P_.push_back(b.pressure);
        }
        mdelast_driver *d = nullptr;
        check_ni(mdelast_batch_create(cfg.data(), static_cast<int32_t>(R), &d));
        d_ = d;
        n_rg_ = rg.size();
    }
    ~BatchedMDDriver() { mdelast_driver_destroy(d_); }
    BatchedMDDriver(BatchedMDDriver const &) = delete;
    BatchedMDDriver &operator=(BatchedMDDriver const &) = delete;

    int n_replicas() const { return static_cast<int>(counts_.size()); }
    long n_atoms() const {
        long s = 0;
        for (size_t n : counts_)
            s += static_cast<long>(n);
        return s;
    }
    double run(int n, int rebuild_every, int sample_every, bool timed) {
        float ms = 0.f;
        check(mdelast_driver_run(d_, n, rebuild_every, sample_every, timed ? &ms : nullptr));
        return ms;
    }
    void integrate() { check(mdelast_driver_integrate(d_, 1)); }
    void calculate_neighbors() { check_ni(mdelast_driver_calculate_neighbors(d_)); }
    void set_sample(bool f) { check(mdelast_driver_set_sample_observables(d_, f ? 1 : 0)); }
    bool get_sample() const {
        int32_t f = 0;
        check(mdelast_driver_get_sample_observables(d_, &f));
        return f != 0;
    }
    py::dict observables(int r) {
        mdelast_observables o;
        check(mdelast_batch_get_observables(d_, r, &o));
        return obs_dict(o);
    }
    py::dict observables_all() {
        std::vector<mdelast_observables> o(static_cast<size_t>(n_replicas()));
        for (int r = 0; r < n_replicas(); ++r)
            check(mdelast_batch_get_observables(d_, r, &o[static_cast<size_t>(r)]));
        return obs_dict_all(o);
    }
    py::array_t<uint32_t> status() {
        py::array_t<uint32_t> a(static_cast<size_t>(n_replicas()));
        check(mdelast_batch_get_status(d_, a.mutable_data()));
        return a;
    }
    // replica r's half list (md_driver.cpp:279-298) as CSR (point, neighbors)
    py::tuple neighbor_list(int r) {
        if (r < 0 || r >= n_replicas())
            throw py::index_error("replica index out of range");
        size_t const N = counts_[static_cast<size_t>(r)];
        py::array_t<int32_t> point(N + 1);
        int64_t total = 0;
        check(mdelast_batch_get_neighbors(d_, r, point.mutable_data(), nullptr, 0, &total));
        py::array_t<int32_t> nb(static_cast<size_t>(total));
        check(mdelast_batch_get_neighbors(d_, r, point.mutable_data(), nb.mutable_data(), total,
                                          &total));
        return py::make_tuple(point, nb);
    }
    py::array_t<double> atoms(int r, int field) {
        if (r < 0 || r >= n_replicas())
            throw py::index_error("replica index out of range");
        size_t const N = counts_[static_cast<size_t>(r)];
        bool const three = field <= MDELAST_ATOM_FORCES;
        py::array_t<double> a = three ? py::array_t<double>({N, size_t(3)}) : py::array_t<double>(N);
        check(mdelast_batch_get_atoms(d_, r, field, a.mutable_data()));
        return a;
    }
    std::vector<double> kernel_times(int n) {
        std::vector<double> t(MDELAST_N_KERNEL_TIMES);
        check(mdelast_driver_kernel_times(d_, n, t.data()));
        return t;
    }
    void synchronize() { check(mdelast_driver_synchronize(d_)); }
    // g(r) of one replica (mode as MDDriver's three calculate_* methods: 0, 1, 2);
    // returns (gr, gr_partial) with gr_partial one row per type pair a <= b
    void set_sample_ring(int capacity) { check(mdelast_driver_set_sample_ring(d_, capacity)); }
    py::dict autotune(int n_repeat) { return autotune_dict(d_, n_repeat); }
    py::dict autotune_steps(int n, int rebuild_every) {
        return autotune_dict(d_, n, rebuild_every);
    }
    py::object force_staging() { return force_staging_get(d_); }
    py::tuple list_capacity() {
        int32_t m = 0, g = 0;
        check(mdelast_driver_list_capacity(d_, &m, &g));
        return py::make_tuple(m, g);
    }
    void set_force_staging(bool on) { check(mdelast_driver_set_force_staging(d_, on ? 1 : 0)); }
    void set_launch(int td, int tf, int bd, int bf) {
        check(mdelast_driver_set_launch(d_, td, tf, bd, bf));
    }
    void set_pair_list(double f) { check(mdelast_driver_set_pair_list(d_, f)); }
    // thermostat (which = 0) or barostat (1) chain of replica r: (q, p_eta, eta)
    py::tuple chain(int r, int which) {
        double q[16], p[16], e[16];
        int32_t n = 0;
        check(mdelast_batch_get_chain(d_, r, which, q, p, e, &n));
        return py::make_tuple(std::vector<double>(q, q + n), std::vector<double>(p, p + n),
                              std::vector<double>(e, e + n));
    }
    py::dict drain_samples(int r) {
        if (r < 0 || r >= n_replicas())
            throw py::index_error("replica index out of range");
        return drain_dict(d_, r);
    }
    void fluctuation_start() { check(mdelast_driver_fluct_start(d_)); }
    mdelast_fluct fluct(int r) {
        mdelast_fluct f;
        check(mdelast_batch_get_fluct(d_, r, &f));
        return f;
    }
    py::dict fluctuations(int r) { return fluct_dict(fluct(r)); }
    py::dict elastic_constants(int r, py::object T, py::object P) {
        if (r < 0 || r >= n_replicas())
            throw py::index_error("replica index out of range");
        size_t const k = static_cast<size_t>(r);
        return elastic_dict(fluct(r), ens_[k], T.is_none() ? T_[k] : T.cast<double>(),
                            P.is_none() ? P_[k] : P.cast<double>());
    }
    py::tuple pair_correlation(int r, int mode) {
        if (r < 0 || r >= n_replicas())
            throw py::index_error("replica index out of range");
        check(mdelast_batch_pair_correlation(d_, r, mode));
        size_t const nt = mass_.size(), np = nt * (nt + 1) / 2;
        py::array_t<double> g(n_rg_), gp({np, n_rg_});
        check(mdelast_batch_get_gr(d_, r, g.mutable_data(), gp.mutable_data()));
        return py::make_tuple(g, gp);
    }

  private:
    mdelast_driver *d_ = nullptr;
    size_t n_rg_ = 0;
    std::vector<int> ens_;
    std::vector<double> T_, P_; // thermostat temperature and barostat pressure per replica
    std::vector<PotentialPtr> pot_;
    std::vector<EAMPtr> eam_;
    std::vector<double> mass_;
    std::vector<size_t> counts_;
};

} // namespace

PYBIND11_MAKE_OPAQUE(std::vector<PotentialPtr>);
PYBIND11_MAKE_OPAQUE(std::vector<EAMPtr>);

PYBIND11_MODULE(md_driver_module, m) {
    m.doc() = "mdelast md driver: B200 path (CUDA kernels behind libmdelast_cuda.so)";

    py::class_<Vector3d, std::shared_ptr<Vector3d>>(m, "Vector3d")
        .def(py::init<double, double, double>())
        .def_readwrite("x", &Vector3d::x)
        .def_readwrite("y", &Vector3d::y)
        .def_readwrite("z", &Vector3d::z)
        .def("length", &Vector3d::length)
        .def("length2", &Vector3d::length2)
        .def("__repr__", [](Vector3d const &v) {
            return "(" + std::to_string(v.x) + "," + std::to_string(v.y) + "," +
                   std::to_string(v.z) + ")";
        });

    py::class_<PotentialValue, std::shared_ptr<PotentialValue>>(m, "PotentialValue")
        .def_readonly("V", &PotentialValue::V)
        .def_readonly("dVdr", &PotentialValue::dVdr)
        .def_readonly("d2Vdr2", &PotentialValue::d2Vdr2);

    py::class_<Potential, std::shared_ptr<Potential>>(m, "Potential")
        .def_readonly("rcut", &Potential::rcut)
        .def("calculate", &Potential::calculate);

    py::class_<Morse, Potential, std::shared_ptr<Morse>>(m, "Morse")
        .def(py::init<double, double, double, double>())
        .def_readonly("D", &Morse::D)
        .def_readonly("r0", &Morse::r0)
        .def_readonly("alpha", &Morse::alpha);

    py::class_<LennardJones, Potential, std::shared_ptr<LennardJones>>(m, "LennardJones")
        .def(py::init<double, double, double>())
        .def_readonly("epsilon", &LennardJones::epsilon)
        .def_readonly("sigma", &LennardJones::sigma);

    py::class_<TablePotential, Potential, std::shared_ptr<TablePotential>>(m, "TablePotential")
        .def(py::init<double, double, double, std::vector<double> const &,
                      std::vector<double> const &, std::vector<double> const &>())
        .def(py::init<double, double, double, std::vector<double> const &,
                      std::vector<double> const &, std::vector<double> const &,
                      std::string const &>())
        .def_readonly("interpolation", &TablePotential::interpolation);

    py::class_<EAM, std::shared_ptr<EAM>>(m, "EAM")
        .def(py::init<double, double, double, double, std::vector<double> const &,
                      std::vector<double> const &, std::vector<double> const &,
                      std::vector<double> const &, std::vector<double> const &,
                      std::vector<double> const &>())
        .def(py::init<double, double, double, double, std::vector<double> const &,
                      std::vector<double> const &, std::vector<double> const &,
                      std::vector<double> const &, std::vector<double> const &,
                      std::vector<double> const &, std::string const &>())
        .def_readonly("interpolation", &EAM::interpolation)
        .def_readonly("rcut", &EAM::rcut)
        .def_readonly("rhomax_fatal", &EAM::rhomax_fatal)
        .def("rho", [](EAM const &e, double r) { return e.eval(0, r); })
        .def("drhodr", [](EAM const &e, double r) { return e.eval(1, r); })
        .def("d2rhodr2", [](EAM const &e, double r) { return e.eval(2, r); })
        .def("F", [](EAM const &e, double r) { return e.eval(3, r); })
        .def("dFdrho", [](EAM const &e, double r) { return e.eval(4, r); })
        .def("d2Fdrho2", [](EAM const &e, double r) { return e.eval(5, r); });

    py::bind_vector<std::vector<PotentialPtr>>(m, "PotentialVector");
    py::bind_vector<std::vector<EAMPtr>>(m, "EAMVector");

    py::class_<MDDriver, std::shared_ptr<MDDriver>> md(m, "MDDriver");
    md.def(py::init<std::vector<Vector3d> const &, std::vector<Vector3d> const &,
                    std::vector<PotentialPtr> const &, std::vector<EAMPtr> const &, Ensamble,
                    ThermostatCoupling, Thermostat const &, Barostat const &, Box const &,
                    std::vector<double> const &, double, std::vector<double> const &,
                    std::vector<unsigned> const &, double, bool, double, double,
                    std::string const &, int>(),
           py::arg("positions"), py::arg("velocities"), py::arg("pot"), py::arg("eam"),
           py::arg("ensamble"), py::arg("thermostat_coupling"), py::arg("thermostat"),
           py::arg("barostat"), py::arg("box"), py::arg("rg"), py::arg("Nf"), py::arg("mass"),
           py::arg("types"), py::arg("dt_global"), py::arg("neighbors"), py::arg("r_skin"),
           py::arg("fatal_conservation"), py::kw_only(), py::arg("precision") = "",
           py::arg("device") = 0)
        .def_property_readonly("positions", [](MDDriver &d) { return d.atoms3(MDELAST_ATOM_POSITIONS); })
        .def_property_readonly("coordinates", [](MDDriver &d) { return d.atoms3(MDELAST_ATOM_COORDINATES); })
        .def_property_readonly("velocities", [](MDDriver &d) { return d.atoms3(MDELAST_ATOM_VELOCITIES); })
        .def_property_readonly("forces", [](MDDriver &d) { return d.atoms3(MDELAST_ATOM_FORCES); })
        .def_property_readonly("rho_eam", [](MDDriver &d) { return d.atoms1(MDELAST_ATOM_RHO); })
        .def_property_readonly("energies_pot", [](MDDriver &d) { return d.atoms1(MDELAST_ATOM_EPOT); })
        .def_property_readonly("energies_kin", [](MDDriver &d) { return d.atoms1(MDELAST_ATOM_EKIN); })
        .def_readonly("ensamble", &MDDriver::ensamble)
        .def_readonly("thermostat_coupling", &MDDriver::thermostat_coupling)
        .def_property_readonly("thermostat", &MDDriver::thermostat)
        .def_property_readonly("barostat", &MDDriver::barostat)
        .def_readonly("box_initial", &MDDriver::box_initial)
        .def_property_readonly("box", &MDDriver::box)
        .def_property_readonly("epot_eam_atom", [](MDDriver &d) { return d.obs().epot_eam_atom; })
        .def_property_readonly("epot_atom", [](MDDriver &d) { return d.obs().epot_atom; })
        .def_property_readonly("ekin_atom", [](MDDriver &d) { return d.obs().ekin_atom; })
        .def_property_readonly("etot_atom", [](MDDriver &d) { return d.obs().etot_atom; })
        .def_property_readonly("etot_cons", [](MDDriver &d) { return d.obs().etot_cons; })
        .def_property_readonly("etot_cons_err", [](MDDriver &d) { return d.obs().etot_cons_err; })
        .def_property_readonly("born_stress_tensor", [](MDDriver &d) { return vec6(d.obs().born_stress_tensor); })
        .def_property_readonly("born_elasticity_tensor", [](MDDriver &d) {
            py::array_t<double> a({6, 6});
            std::copy(d.obs().born_elasticity_tensor, d.obs().born_elasticity_tensor + 36, a.mutable_data());
            return a;
        })
        .def_property_readonly("temperature_kin", [](MDDriver &d) { return d.obs().temperature_kin; })
        .def_property_readonly("temperature_conf_inverse", [](MDDriver &d) { return d.obs().temperature_conf_inverse; })
        .def_property_readonly("total_laplacian", [](MDDriver &d) { return d.obs().total_laplacian; })
        .def_property_readonly("total_force2", [](MDDriver &d) { return d.obs().total_force2; })
        .def_property_readonly("pressure", [](MDDriver &d) { return d.obs().pressure; })
        .def_property_readonly("stress_tensor", [](MDDriver &d) { return vec6(d.obs().stress_tensor); })
        .def_readonly("dt_global", &MDDriver::dt_global)
        .def_property_readonly("time", [](MDDriver &d) { return d.obs().time; })
        .def_property_readonly("cycle", [](MDDriver &d) { return static_cast<unsigned long long>(d.obs().cycle); })
        .def_readonly("rg", &MDDriver::rg)
        .def_readonly("gr", &MDDriver::gr)
        .def_readonly("gr_partial", &MDDriver::gr_partial)
        .def_readonly("fatal_conservation", &MDDriver::fatal_conservation)
        .def_property("sample_observables", &MDDriver::get_sample, &MDDriver::set_sample)
        .def_readonly("mass", &MDDriver::mass)
        .def_readonly("types", &MDDriver::types)
        .def_readonly("Nparticles_per_type", &MDDriver::Nparticles_per_type)
        .def("integrate", &MDDriver::integrate)
        .def("calculate_neighbors", &MDDriver::calculate_neighbors)
        .def("calculate_pair_correlation", [](MDDriver &d) { d.pair_correlation(0); })
        .def("calculate_pair_correlations", [](MDDriver &d) { d.pair_correlation(1); })
        .def("calculate_partial_pair_correlation", [](MDDriver &d) { d.pair_correlation(2); })
        .def("autotune", &MDDriver::autotune, py::arg("n_repeat") = 3,
             "time the pair passes over their launch shapes and keep the fastest")
        .def("autotune_steps", &MDDriver::autotune_steps, py::arg("n_steps") = 4,
             py::arg("rebuild_every") = 20,
             "the same on real steps (the state advances by about 30 n_steps steps)")
        .def("set_launch", &MDDriver::set_launch, py::arg("tpa_density"), py::arg("tpa_force"),
             py::arg("blocks_density"), py::arg("blocks_force"))
        .def_property("force_staging", &MDDriver::force_staging, &MDDriver::set_force_staging,
                      "force pass reading shared-memory tables (None: no staged copy)")
        .def_property_readonly("list_capacity", &MDDriver::list_capacity,
                               "(neighbour slots per atom, launches resumed after a list overflow)")
        .def("set_pair_list", &MDDriver::set_pair_list, py::arg("factor"),
             "pair passes walk the list's pairs within factor * r_cut (0: the full list)")
        .def("set_sample_ring", &MDDriver::set_sample_ring, py::arg("capacity"),
             "room for this many sampled steps between drains (0: no ring)")
        .def("drain_samples", &MDDriver::drain_samples,
             "records of the sampled steps since the last drain, as arrays")
        .def("fluctuation_start", &MDDriver::fluctuation_start,
             "clear the fluctuation sums and accumulate from the next sampled step")
        .def("fluctuations", &MDDriver::fluctuations)
        .def("elastic_constants", &MDDriver::elastic_constants, py::arg("T") = py::none(),
             py::arg("P") = py::none(),
             "the fluctuation estimate of C_ij from the accumulated sums (defaults: the "
             "thermostat temperature and barostat pressure)")
        // additions of the B200 path
        .def("integrate_n", &MDDriver::integrate_n, py::arg("n_steps"))
        .def("atoms_array", &MDDriver::atoms_array, py::arg("field"))
        .def("neighbor_list", &MDDriver::neighbor_list)
        .def("synchronize", &MDDriver::synchronize)
        .def("run", &MDDriver::run, py::arg("n_steps"), py::arg("rebuild_every") = 20,
             py::arg("sample_every") = 1, py::arg("timed") = false,
             "n_steps of the molecular_dynamics.py run loop on the device (list rebuild every "
             "rebuild_every steps, observables every sample_every steps); returns the device "
             "time in ms when timed")
        .def("kernel_times", &MDDriver::kernel_times, py::arg("n_steps") = 10,
             "mean device ms per launch: opening scalar, kick+drift, density, force, closing "
             "scalar, list build")
        .def_readonly("precision", &MDDriver::precision_)
        .def_property_readonly("status", [](MDDriver &d) { return d.obs().status; });

    py::class_<BatchedMDDriver, std::shared_ptr<BatchedMDDriver>>(m, "BatchedMDDriver")
        .def(py::init<std::vector<py::array_t<double, py::array::c_style | py::array::forcecast>> const &,
                      std::vector<py::array_t<double, py::array::c_style | py::array::forcecast>> const &,
                      std::vector<py::array_t<uint32_t, py::array::c_style | py::array::forcecast>> const &,
                      std::vector<PotentialPtr> const &,
                      std::vector<EAMPtr> const &, std::vector<Ensamble> const &,
                      std::vector<Thermostat> const &, std::vector<Barostat> const &,
                      std::vector<Box> const &, std::vector<double> const &,
                      std::vector<double> const &, double, bool, double, double,
                      std::string const &, int, std::vector<double> const &>(),
             py::arg("positions"), py::arg("velocities"), py::arg("types"), py::arg("pot"),
             py::arg("eam"), py::arg("ensembles"), py::arg("thermostats"), py::arg("barostats"),
             py::arg("boxes"), py::arg("Nf"), py::arg("mass"), py::arg("dt_global"),
             py::arg("neighbors") = true, py::arg("r_skin") = 1.2,
             py::arg("fatal_conservation") = 1e3, py::arg("precision") = "",
             py::arg("device") = 0,
             py::arg("rg") = std::vector<double>{1e-10, 2e-10})
        .def_property_readonly("n_replicas", &BatchedMDDriver::n_replicas)
        .def_property_readonly("n_atoms", &BatchedMDDriver::n_atoms)
        .def("run", &BatchedMDDriver::run, py::arg("n_steps"), py::arg("rebuild_every") = 20,
             py::arg("sample_every") = 1, py::arg("timed") = false)
        .def("integrate", &BatchedMDDriver::integrate)
        .def("calculate_neighbors", &BatchedMDDriver::calculate_neighbors)
        .def_property("sample_observables", &BatchedMDDriver::get_sample, &BatchedMDDriver::set_sample)
        .def("observables", &BatchedMDDriver::observables, py::arg("replica"))
        .def("observables_all", &BatchedMDDriver::observables_all)
        .def("status", &BatchedMDDriver::status)
        .def("atoms", &BatchedMDDriver::atoms, py::arg("replica"), py::arg("field"))
        .def("neighbor_list", &BatchedMDDriver::neighbor_list, py::arg("replica"))
        .def("kernel_times", &BatchedMDDriver::kernel_times, py::arg("n_steps") = 10)
        .def("autotune", &BatchedMDDriver::autotune, py::arg("n_repeat") = 3)
        .def("autotune_steps", &BatchedMDDriver::autotune_steps, py::arg("n_steps") = 4,
             py::arg("rebuild_every") = 20)
        .def("set_launch", &BatchedMDDriver::set_launch, py::arg("tpa_density"),
             py::arg("tpa_force"), py::arg("blocks_density"), py::arg("blocks_force"))
        .def_property("force_staging", &BatchedMDDriver::force_staging,
                      &BatchedMDDriver::set_force_staging)
        .def_property_readonly("list_capacity", &BatchedMDDriver::list_capacity)
        .def("set_pair_list", &BatchedMDDriver::set_pair_list, py::arg("factor"))
        .def("set_sample_ring", &BatchedMDDriver::set_sample_ring, py::arg("capacity"))
        .def("drain_samples", &BatchedMDDriver::drain_samples, py::arg("replica"))
        .def("chain", &BatchedMDDriver::chain, py::arg("replica"), py::arg("which") = 0)
        .def("fluctuation_start", &BatchedMDDriver::fluctuation_start)
        .def("fluctuations", &BatchedMDDriver::fluctuations, py::arg("replica"))
        .def("elastic_constants", &BatchedMDDriver::elastic_constants, py::arg("replica"),
             py::arg("T") = py::none(), py::arg("P") = py::none())
        .def("pair_correlation", &BatchedMDDriver::pair_correlation, py::arg("replica"),
             py::arg("mode") = 1)
        .def("synchronize", &BatchedMDDriver::synchronize);

    py::class_<Box, std::shared_ptr<Box>>(m, "Box")
        .def(py::init<py::array_t<double, py::array::c_style | py::array::forcecast>>())
        .def_property_readonly("h", &Box::h_array)
        .def("volume", &Box::volume)
        .def("length", &Box::length);

    py::class_<Thermostat, std::shared_ptr<Thermostat>>(m, "Thermostat")
        .def(py::init<double, std::vector<double>, std::vector<double>, double>())
        .def_readonly("temperature", &Thermostat::temperature)
        .def_readonly("q", &Thermostat::q)
        .def_readonly("p_eta", &Thermostat::p_eta)
        .def_readonly("eta", &Thermostat::eta)
        .def_readonly("nchain", &Thermostat::nchain)
        .def_readonly("Nf", &Thermostat::Nf);

    py::class_<Barostat, std::shared_ptr<Barostat>>(m, "Barostat")
        .def(py::init<double, double, double, Thermostat const &>())
        .def_readonly("pressure", &Barostat::pressure)
        .def_readonly("w", &Barostat::w)
        .def_readonly("epsilon", &Barostat::epsilon)
        .def_readonly("p_epsilon", &Barostat::p_epsilon)
        .def_readonly("thermostat", &Barostat::thermostat);

    py::class_<BarostatFlex, std::shared_ptr<BarostatFlex>>(m, "BarostatFlex")
        .def(py::init<double, double, py::array_t<double>, Thermostat const &>())
        .def_readonly("pressure", &BarostatFlex::pressure)
        .def_readonly("w", &BarostatFlex::w)
        .def_readonly("pg", &BarostatFlex::pg)
        .def_readonly("thermostat", &BarostatFlex::thermostat);

    py::enum_<Ensamble>(md, "Ensamble")
        .value("NVE", NVE)
        .value("NVT", NVT)
        .value("NPT", NPT)
        .value("NPT_FLEX", NPT_FLEX)
        .export_values();

    py::enum_<ThermostatCoupling>(md, "ThermostatCoupling")
        .value("THERMOSTAT_KINETIC", THERMOSTAT_KINETIC)
        .value("THERMOSTAT_CONFIGURATIONAL", THERMOSTAT_CONFIGURATIONAL)
        .value("THERMOSTAT_AVERAGE", THERMOSTAT_AVERAGE)
        .export_values();

    // units.hpp:6-24
    struct UnitsTag {};
    py::class_<UnitsTag> units(m, "Units");
    units.attr("k_boltz") = 1.38064852e-16;
    units.attr("Navogadro") = 6.02214086e23;
    units.attr("ev") = 1.6021773e-12;
    units.attr("joule") = 1e7;
    units.attr("angstrom") = kAngstrom;
    units.attr("nm") = 1e-7;
    units.attr("bar") = 1e6;
    units.attr("kbar") = 1e3 * 1e6;
    units.attr("atm") = 1.01325 * 1e6;
    units.attr("Pa") = 1e-5 * 1e6;
    units.attr("GPa") = 1e9 * (1e-5 * 1e6);
    units.attr("mus") = 1e-6;
    units.attr("ns") = 1e-9;
    units.attr("ps") = 1e-12;
    units.attr("fs") = 1e-15;

    m.def("device_available", []() { return mdelast_device_available() != 0; });
    m.def("release_cached_memory", [](int device) { check(mdelast_release_cached_memory(device)); },
          py::arg("device") = 0);
    m.def("set_default_precision", [](std::string const &p) {
        if (p != "fp64" && p != "mixed")
            throw py::value_error("precision must be 'fp64' or 'mixed'");
        default_precision = p;
    });
    m.attr("ATOM_POSITIONS") = MDELAST_ATOM_POSITIONS;
    m.attr("ATOM_COORDINATES") = MDELAST_ATOM_COORDINATES;
    m.attr("ATOM_VELOCITIES") = MDELAST_ATOM_VELOCITIES;
    m.attr("ATOM_FORCES") = MDELAST_ATOM_FORCES;
    m.attr("ATOM_RHO") = MDELAST_ATOM_RHO;
    m.attr("ATOM_EPOT") = MDELAST_ATOM_EPOT;
    m.attr("ATOM_EKIN") = MDELAST_ATOM_EKIN;
}
