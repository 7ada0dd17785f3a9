// file_io.cpp -- the reference's binary state file (src/file_io.cpp:29-490):
// little-endian, packed, no header.  Field order:
//   nd i32, np u32; dt, current, total, file_dt f64; step_count u32;
//   origo[3], L[3] f64; num[3] u32; periodic i32;
//   per particle x,y,z,r | xysum[2] | vel,fixvel | force[3] | angpos[3] |
//   angvel[3] | torque[3] (each array for all particles in turn);
//   es_dot, es, ev_dot, ev, p (np each);
//   g[3], k_n, k_t, k_r, gamma_n, gamma_t, gamma_r, mu_s, mu_d, mu_r,
//   gamma_wn, gamma_wt, mu_ws, mu_wd, rho f64; contactmodel u32;
//   kappa, db, V_b f64; nw u32, wmode[nw] i32, (n[3], pos) per wall,
//   (m, vel, force, devs) per wall, devs_A, devs_f f64;
//   lambda_bar f64, nb0 u32, sigma_b, tau_b f64, bonds (u32,u32)*nb0,
//   delta_n[nb0], delta_t[nb0][3], omega_n[nb0], omega_t[nb0][3] f64; nu f64;
//   fluid cells when nu > 0: with Darcy flow, per cell (x fastest, then y,
//   then z) V[3], H, phi, K f64 (src/file_io.cpp:270-292, 466-479); without
//   it, kept as opaque bytes.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>

#include "sphere.h"

namespace {

struct In {
    std::vector<char> buf;
    size_t off = 0;
    const char *name;
    template <typename T>
    T get()
    {
        T v{};
        if (off + sizeof(T) > buf.size()) {
            std::cerr << "Error: input binary '" << name << "' is truncated at byte " << off
                      << std::endl;
            exit(1);
        }
        std::memcpy(&v, buf.data() + off, sizeof(T));
        off += sizeof(T);
        return v;
    }
};

struct Out {
    std::ofstream &o;
    template <typename T>
    void put(const T &v)
    {
        o.write(reinterpret_cast<const char *>(&v), sizeof(T));
    }
};

}  // namespace

void DEM::readbin(const char *target)
{
    std::ifstream ifs(target, std::ios_base::binary);
    if (!ifs) {
        std::cerr << "Could not read input binary file '" << target << "'" << std::endl;
        exit(1);
    }
    In in{std::vector<char>(std::istreambuf_iterator<char>(ifs), std::istreambuf_iterator<char>()), 0,
          target};
    const int32_t nd = in.get<int32_t>();
    const uint32_t np = in.get<uint32_t>();
    if (nd != 3) {
        std::cerr << "Dimensionality mismatch between dataset and this SPHERE program.\n"
                  << "The dataset is " << nd << "D, this SPHERE binary is 3D.\n"
                  << "This execution is terminating." << std::endl;
        exit(-1);
    }
    cfg_ = sph_config{};
    cfg_.np = np;
    dt_ = in.get<double>();
    current_ = in.get<double>();
    total_ = in.get<double>();
    file_dt_ = in.get<double>();
    step_count_ = in.get<uint32_t>();
    cfg_.dt = dt_;
    for (double &v : cfg_.origo) v = in.get<double>();
    for (double &v : cfg_.L) v = in.get<double>();
    for (uint32_t &v : cfg_.num) v = in.get<uint32_t>();
    cfg_.periodic = in.get<int32_t>();
    const size_t n = np;
    x_.assign(4 * n, 0.0);
    xysum_.assign(2 * n, 0.0);
    vel_.assign(4 * n, 0.0);
    force_.assign(4 * n, 0.0);
    angpos_.assign(4 * n, 0.0);
    angvel_.assign(4 * n, 0.0);
    torque_.assign(4 * n, 0.0);
    for (size_t i = 0; i < 4 * n; ++i) x_[i] = in.get<double>();
    for (size_t i = 0; i < 2 * n; ++i) xysum_[i] = in.get<double>();
    for (size_t i = 0; i < 4 * n; ++i) vel_[i] = in.get<double>();
    for (auto *a : {&force_, &angpos_, &angvel_, &torque_})
        for (size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) (*a)[4 * i + k] = in.get<double>();
    for (auto *a : {&es_dot_, &es_, &ev_dot_, &ev_, &p_}) {
        a->assign(n, 0.0);
        for (size_t i = 0; i < n; ++i) (*a)[i] = in.get<double>();
    }
    for (double &v : cfg_.g) v = in.get<double>();
    for (double *v : {&cfg_.k_n, &cfg_.k_t, &cfg_.k_r, &cfg_.gamma_n, &cfg_.gamma_t,
                      &cfg_.gamma_r, &cfg_.mu_s, &cfg_.mu_d, &cfg_.mu_r, &cfg_.gamma_wn,
                      &cfg_.gamma_wt, &cfg_.mu_ws, &cfg_.mu_wd, &cfg_.rho})
        *v = in.get<double>();
    cfg_.contactmodel = in.get<uint32_t>();
    cfg_.kappa = in.get<double>();
    cfg_.db = in.get<double>();
    cfg_.V_b = in.get<double>();
    cfg_.nw = in.get<uint32_t>();
    if (cfg_.nw > SPHK_MAXWALLS) {
        std::cerr << "Error; MAXWALLS (" << SPHK_MAXWALLS << ") in datatypes.h "
                  << "is smaller than the number of walls specified in the "
                  << "input file (" << cfg_.nw << ").\n";
        exit(1);
    }
    for (uint32_t w = 0; w < cfg_.nw; ++w) cfg_.wmode[w] = in.get<int32_t>();
    walls_nx_.assign(4 * cfg_.nw, 0.0);
    walls_mvfd_.assign(4 * cfg_.nw, 0.0);
    for (double &v : walls_nx_) v = in.get<double>();
    for (double &v : walls_mvfd_) v = in.get<double>();
    cfg_.devs_A = in.get<double>();
    cfg_.devs_f = in.get<double>();
    cfg_.lambda_bar = in.get<double>();
    cfg_.nb0 = in.get<uint32_t>();
    cfg_.sigma_b = in.get<double>();
    cfg_.tau_b = in.get<double>();
    const size_t nb = cfg_.nb0;
    bonds_.assign(2 * nb, 0u);
    bonds_delta_.assign(4 * nb, 0.0);
    bonds_omega_.assign(4 * nb, 0.0);
    for (uint32_t &v : bonds_) v = in.get<uint32_t>();
    for (size_t b = 0; b < nb; ++b) bonds_delta_[4 * b + 3] = in.get<double>();
    for (size_t b = 0; b < nb; ++b)
        for (int k = 0; k < 3; ++k) bonds_delta_[4 * b + k] = in.get<double>();
    for (size_t b = 0; b < nb; ++b) bonds_omega_[4 * b + 3] = in.get<double>();
    for (size_t b = 0; b < nb; ++b)
        for (int k = 0; k < 3; ++k) bonds_omega_[4 * b + k] = in.get<double>();
    nu_ = in.get<double>();
    fluid_trailer_.clear();
    if (darcyOn()) {
        initDarcyMem();
        for (uint32_t z = 0; z < cfg_.num[2]; ++z)
            for (uint32_t y = 0; y < cfg_.num[1]; ++y)
                for (uint32_t x = 0; x < cfg_.num[0]; ++x) {
                    const size_t i = darcyNode((int)x, (int)y, (int)z);
                    for (int k = 0; k < 3; ++k) d_V_[3 * i + k] = in.get<double>();
                    d_H_[i] = in.get<double>();
                    d_phi_[i] = in.get<double>();
                    d_K_[i] = in.get<double>();
                }
    } else {
        fluid_trailer_.assign(in.buf.begin() + (std::ptrdiff_t)in.off, in.buf.end());
    }
}

void DEM::writebin(const char *target)
{
    std::ofstream ofs(target, std::ios_base::binary);
    if (!ofs) {
        std::cerr << "could create output binary file '" << target << std::endl;
        exit(1);
    }
    Out o{ofs};
    o.put<int32_t>(3);
    o.put<uint32_t>(cfg_.np);
    o.put(dt_);
    o.put(current_);
    o.put(total_);
    o.put(file_dt_);
    o.put(step_count_);
    for (double v : cfg_.origo) o.put(v);
    for (double v : cfg_.L) o.put(v);
    for (uint32_t v : cfg_.num) o.put(v);
    o.put<int32_t>(cfg_.periodic);
    const size_t n = cfg_.np;
    for (size_t i = 0; i < 4 * n; ++i) o.put(x_[i]);
    for (size_t i = 0; i < 2 * n; ++i) o.put(xysum_[i]);
    for (size_t i = 0; i < 4 * n; ++i) o.put(vel_[i]);
    for (auto *a : {&force_, &angpos_, &angvel_, &torque_})
        for (size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) o.put((*a)[4 * i + k]);
    for (auto *a : {&es_dot_, &es_, &ev_dot_, &ev_, &p_})
        for (size_t i = 0; i < n; ++i) o.put((*a)[i]);
    for (double v : cfg_.g) o.put(v);
    for (double v : {cfg_.k_n, cfg_.k_t, cfg_.k_r, cfg_.gamma_n, cfg_.gamma_t, cfg_.gamma_r,
                     cfg_.mu_s, cfg_.mu_d, cfg_.mu_r, cfg_.gamma_wn, cfg_.gamma_wt, cfg_.mu_ws,
                     cfg_.mu_wd, cfg_.rho})
        o.put(v);
    o.put(cfg_.contactmodel);
    o.put(cfg_.kappa);
    o.put(cfg_.db);
    o.put(cfg_.V_b);
    o.put(cfg_.nw);
    for (uint32_t w = 0; w < cfg_.nw; ++w) o.put<int32_t>(cfg_.wmode[w]);
    for (double v : walls_nx_) o.put(v);
    for (double v : walls_mvfd_) o.put(v);
    o.put(cfg_.devs_A);
    o.put(cfg_.devs_f);
    o.put(cfg_.lambda_bar);
    o.put(cfg_.nb0);
    o.put(cfg_.sigma_b);
    o.put(cfg_.tau_b);
    for (uint32_t v : bonds_) o.put(v);
    const size_t nb = cfg_.nb0;
    for (size_t b = 0; b < nb; ++b) o.put(bonds_delta_[4 * b + 3]);
    for (size_t b = 0; b < nb; ++b)
        for (int k = 0; k < 3; ++k) o.put(bonds_delta_[4 * b + k]);
    for (size_t b = 0; b < nb; ++b) o.put(bonds_omega_[4 * b + 3]);
    for (size_t b = 0; b < nb; ++b)
        for (int k = 0; k < 3; ++k) o.put(bonds_omega_[4 * b + k]);
    o.put(nu_);
    if (darcyOn()) {
        for (uint32_t z = 0; z < cfg_.num[2]; ++z)
            for (uint32_t y = 0; y < cfg_.num[1]; ++y)
                for (uint32_t x = 0; x < cfg_.num[0]; ++x) {
                    const size_t i = darcyNode((int)x, (int)y, (int)z);
                    for (int k = 0; k < 3; ++k) o.put(d_V_[3 * i + k]);
                    o.put(d_H_[i]);
                    o.put(d_phi_[i]);
                    o.put(d_K_[i]);
                }
    } else if (!fluid_trailer_.empty()) {
        ofs.write(fluid_trailer_.data(), (std::streamsize)fluid_trailer_.size());
    }
}
