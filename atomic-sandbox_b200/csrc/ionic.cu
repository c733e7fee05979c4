// ionic.cu -- host side of the pseudopotential terms: the ionic setup of a solver (the species tables
// copied to the device), the per-geometry centres and projector spheres (the ball of each projector as
// a clipped box of grid points, crates/qm/src/nuclear.rs:320-336 points_within), and the nonlocal
// operator's apply, projection and force sums over the kernels of k_ionic.cu.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include "solver.h"

namespace ks {

namespace {

void grow(DevBuf& b, size_t bytes) {
    if (b.bytes < bytes) b.alloc(bytes);
}

bool finite_table(const double* t, int n) {
    if (n > 0 && !t) return false;
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(t[i])) return false;
    return true;
}

}  // namespace

void Ionic::set(const ks_species* sp, int nsp) {
    if (nsp < 0 || nsp > MAX_SPECIES) throw std::invalid_argument("ionic setup: 0..8 species");
    if (nsp > 0 && !sp) throw std::invalid_argument("ionic setup: species is NULL");
    std::vector<Species> out;
    for (int i = 0; i < nsp; ++i) {
        const ks_species& s = sp[i];
        const std::string who = "ionic setup, species Z=" + std::to_string(s.z) + ": ";
        if (s.z < 1 || s.z > 118) throw std::invalid_argument(who + "atomic number out of range");
        for (const auto& o : out)
            if (o.z == s.z) throw std::invalid_argument(who + "listed twice");
        if (!(std::isfinite(s.z_v) && s.z_v > 0.0)) throw std::invalid_argument(who + "z_v must be > 0");
        if (!(std::isfinite(s.sigma_lr) && s.sigma_lr > 0.0)) throw std::invalid_argument(who + "sigma_lr must be > 0");
        if (!(std::isfinite(s.du) && s.du > 0.0)) throw std::invalid_argument(who + "du must be > 0");
        // every radius spans at most 1e9 table steps (the reads index the table by d / du)
        auto span_ok = [&](double r) { return std::isfinite(r) && r / s.du < 1e9; };
        if (!span_ok(s.r_sr) || !span_ok(s.pc_radius)) throw std::invalid_argument(who + "a radius is not finite or spans over 1e9 table steps");
        for (int k = 0; k < s.n_proj && s.proj_radius; ++k)
            if (!span_ok(s.proj_radius[k])) throw std::invalid_argument(who + "a projector radius spans over 1e9 table steps");
        if (s.n_v_sr < 0 || (s.n_v_sr > 0 && s.n_v_sr < 4) || !finite_table(s.v_sr, s.n_v_sr) || (s.n_v_sr > 0 && !(s.r_sr >= 0.0)))
            throw std::invalid_argument(who + "V_SR table: n = 0 or >= 4 finite values and r_sr >= 0");
        const bool core = s.pc_radius > 0.0;
        if (core && (s.n_rho_pc < 4 || !finite_table(s.rho_pc, s.n_rho_pc)))
            throw std::invalid_argument(who + "partial core: pc_radius > 0 needs >= 4 finite table values");
        if (s.n_proj < 0 || s.n_proj > MAX_PROJECTORS || (s.n_proj > 0 && (!s.proj_l || !s.proj_e_kb || !s.proj_radius || !s.proj_t || !s.proj_n)))
            throw std::invalid_argument(who + "0..4 projectors with l, E_KB, radius and table each");
        Species t;
        t.z = s.z;
        t.z_v = s.z_v;
        t.sigma_lr = s.sigma_lr;
        t.du = s.du;
        t.r_sr = s.n_v_sr > 0 ? s.r_sr : 0.0;
        t.v_sr.assign(s.v_sr, s.v_sr + s.n_v_sr);
        t.pc_radius = core ? s.pc_radius : 0.0;
        if (core) t.rho_pc.assign(s.rho_pc, s.rho_pc + s.n_rho_pc);
        for (int k = 0; k < s.n_proj; ++k) {
            if (s.proj_l[k] < 0 || s.proj_l[k] > 2) throw std::invalid_argument(who + "projector l must be 0, 1 or 2");
            if (!std::isfinite(s.proj_e_kb[k]) || !(std::isfinite(s.proj_radius[k]) && s.proj_radius[k] > 0.0) || s.proj_n[k] < 4 ||
                !finite_table(s.proj_t[k], s.proj_n[k]))
                throw std::invalid_argument(who + "projector: finite E_KB, radius > 0, >= 4 finite table values");
            t.proj.push_back({s.proj_l[k], s.proj_e_kb[k], s.proj_radius[k], std::vector<double>(s.proj_t[k], s.proj_t[k] + s.proj_n[k])});
        }
        out.push_back(std::move(t));
    }
    species_ = std::move(out);
    ++gen_;
    // tables: every species' arrays back to back in one device buffer
    std::vector<double> all;
    off_v_sr_.clear();
    off_pc_.clear();
    off_t_.clear();
    for (const auto& t : species_) {
        off_v_sr_.push_back(all.size());
        all.insert(all.end(), t.v_sr.begin(), t.v_sr.end());
        off_pc_.push_back(all.size());
        all.insert(all.end(), t.rho_pc.begin(), t.rho_pc.end());
        off_t_.emplace_back();
        for (const auto& p : t.proj) {
            off_t_.back().push_back(all.size());
            all.insert(all.end(), p.t.begin(), p.t.end());
        }
    }
    if (species_.empty()) return;
    tables_.alloc(std::max<size_t>(all.size(), 1) * sizeof(double));
    KS_CUDA(cudaMemcpy(tables_.p, all.data(), all.size() * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<IonicSpeciesDev> sd;
    for (size_t i = 0; i < species_.size(); ++i) {
        const auto& t = species_[i];
        IonicSpeciesDev d{};
        d.du = t.du;
        d.r_sr = t.r_sr;
        d.pc_radius = t.pc_radius;
        d.v_sr = tables_.d() + off_v_sr_[i];
        d.rho_pc = tables_.d() + off_pc_[i];
        d.n_v_sr = (int)t.v_sr.size();
        d.n_pc = (int)t.rho_pc.size();
        sd.push_back(d);
    }
    species_dev_.alloc(sd.size() * sizeof(IonicSpeciesDev));
    KS_CUDA(cudaMemcpy(species_dev_.p, sd.data(), sd.size() * sizeof(IonicSpeciesDev), cudaMemcpyHostToDevice));
    // a pageable copy may still be in flight when cudaMemcpy returns; the solver's streams do not wait on the
    // legacy stream, so finish the copies before any of their kernels reads the tables
    KS_CUDA(cudaStreamSynchronize(0));
}

int Ionic::species_of(int z) const {
    for (size_t i = 0; i < species_.size(); ++i)
        if (species_[i].z == z) return (int)i;
    return -1;
}

double Ionic::charge_of(int z) const {
    const int i = species_of(z);
    return i < 0 ? (double)z : species_[i].z_v;
}

// crates/qm/src/nuclear.rs:309-315 (centres) and :320-336 (points_within's clipped box); nonlocal.rs build_inner
void Ionic::update(const Layout& L, const ks_nucleus* nuc, int nn, double sigma_ae, cudaStream_t s) {
    if (nn > MAX_CENTRES) throw std::invalid_argument("ionic setup: at most 32 nuclei");
    for (int a = 0; a < nn; ++a)
        for (int ax = 0; ax < 3; ++ax)
            if (!std::isfinite(nuc[a].pos[ax]) || std::fabs(nuc[a].pos[ax]) > 1e6) throw std::invalid_argument("ionic setup: nucleus position not finite");
    centres_h_.clear();
    sph_h_.clear();
    row_ekb_.clear();
    row_ion_.clear();
    chunk_sphere_h_.clear();
    has_core_ = false;
    rows_total_ = 0;
    total_chunks_ = 0;
    max_pts_ = 0;
    long long beta_total = 0;
    int lo_u[3] = {L.n, L.n, L.n}, hi_u[3] = {-1, -1, -1};
    for (int a = 0; a < nn; ++a) {
        const int si = species_of(nuc[a].z);
        IonicCentre c{};
        c.x = nuc[a].pos[0];
        c.y = nuc[a].pos[1];
        c.z = nuc[a].pos[2];
        c.q = si < 0 ? (double)nuc[a].z : species_[si].z_v;
        c.sigma = si < 0 ? sigma_ae : species_[si].sigma_lr;
        c.species = si;
        centres_h_.push_back(c);
        if (si < 0) continue;
        const Species& t = species_[si];
        if (t.pc_radius > 0.0) has_core_ = true;
        for (size_t k = 0; k < t.proj.size(); ++k) {
            const Proj& p = t.proj[k];
            int lo[3], hi[3];
            bool empty = false;
            for (int ax = 0; ax < 3; ++ax) {
                const double l = std::max(std::floor((nuc[a].pos[ax] - p.radius - L.origin) / L.h), 0.0);
                const double h = std::min(std::ceil((nuc[a].pos[ax] + p.radius - L.origin) / L.h), (double)(L.n - 1));
                if (!(h >= l)) { empty = true; break; }
                lo[ax] = (int)l;
                hi[ax] = (int)h;
            }
            if (empty) continue;
            Sphere sp{};
            sp.cx = c.x;
            sp.cy = c.y;
            sp.cz = c.z;
            sp.radius = p.radius;
            sp.e_kb = p.e_kb;
            sp.du = t.du;
            sp.t = tables_.d() + off_t_[si][k];
            sp.n_t = (int)p.t.size();
            sp.l = p.l;
            sp.rows = 2 * p.l + 1;
            sp.row0 = rows_total_;
            sp.i0 = lo[0];
            sp.j0 = lo[1];
            sp.k0 = lo[2];
            sp.ni = hi[0] - lo[0] + 1;
            sp.nj = hi[1] - lo[1] + 1;
            sp.nk = hi[2] - lo[2] + 1;
            const int npts = sp.ni * sp.nj * sp.nk;
            sp.beta0 = beta_total;
            sp.chunks = std::max(1, std::min(MAX_CHUNKS, ceil_div(npts, 1024)));
            sp.chunk0 = total_chunks_;
            for (int q = 0; q < sp.chunks; ++q) chunk_sphere_h_.push_back((int)sph_h_.size());
            total_chunks_ += sp.chunks;
            beta_total += (long long)sp.rows * npts;
            max_pts_ = std::max(max_pts_, npts);
            for (int r = 0; r < sp.rows; ++r) {
                row_ekb_.push_back(p.e_kb);
                row_ion_.push_back(a);
            }
            rows_total_ += sp.rows;
            for (int ax = 0; ax < 3; ++ax) {
                lo_u[ax] = std::min(lo_u[ax], lo[ax]);
                hi_u[ax] = std::max(hi_u[ax], hi[ax]);
            }
            sph_h_.push_back(sp);
        }
    }
    for (int ax = 0; ax < 3; ++ax) {
        ubox_[ax] = sph_h_.empty() ? 0 : lo_u[ax];
        ubox_[3 + ax] = sph_h_.empty() ? 0 : hi_u[ax] - lo_u[ax] + 1;
    }
    grow(centres_, std::max<size_t>(centres_h_.size(), 1) * sizeof(IonicCentre));
    if (!centres_h_.empty())
        KS_CUDA(cudaMemcpyAsync(centres_.p, centres_h_.data(), centres_h_.size() * sizeof(IonicCentre), cudaMemcpyHostToDevice, s));
    if (!sph_h_.empty()) {
        grow(spheres_, sph_h_.size() * sizeof(Sphere));
        grow(chunk_sphere_, chunk_sphere_h_.size() * sizeof(int));
        grow(beta_, (size_t)beta_total * sizeof(float));
        KS_CUDA(cudaMemcpyAsync(spheres_.p, sph_h_.data(), sph_h_.size() * sizeof(Sphere), cudaMemcpyHostToDevice, s));
        KS_CUDA(cudaMemcpyAsync(chunk_sphere_.p, chunk_sphere_h_.data(), chunk_sphere_h_.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        launch_beta(L, static_cast<const Sphere*>(spheres_.p), (int)sph_h_.size(), max_pts_, beta_.f(), s);
    }
    // the host vectors above are read by the copies; keep the stream ordered before they change again
    KS_CUDA(cudaStreamSynchronize(s));
}

void Ionic::local_potential(const Layout& L, float* out, cudaStream_t s) const {
    launch_ionic_local(L, centres(), n_centres(), species_dev(), out, s);
}

void Ionic::partial_core(const Layout& L, float* out, cudaStream_t s) const {
    launch_partial_core(L, centres(), n_centres(), species_dev(), out, s);
}

void Ionic::ensure(Scratch& sc, int count) const {
    const size_t need = (size_t)std::max(count, 1) * std::max(rows_total_, 1);
    if (sc.cap < need) {
        sc.partials.alloc(need * MAX_CHUNKS * 4 * sizeof(double));
        sc.coef.alloc(need * sizeof(double));
        sc.cap = need;
    }
}

void Ionic::apply_nl(const Layout& L, const float* x, int count, float* out, Scratch& sc, cudaStream_t s) const {
    if (sph_h_.empty() || count <= 0) return;
    ensure(sc, count);
    launch_nl_project(L, static_cast<const Sphere*>(spheres_.p), (int)sph_h_.size(), static_cast<const int*>(chunk_sphere_.p),
                      total_chunks_, beta_.f(), x, count, rows_total_, sc.partials.d(), sc.coef.d(), s);
    launch_nl_scatter(L, static_cast<const Sphere*>(spheres_.p), (int)sph_h_.size(), beta_.f(), sc.coef.d(), rows_total_, ubox_, count,
                      out, s);
}

void Ionic::project(const Layout& L, const float* x, int count, Scratch& sc, cudaStream_t s, std::vector<double>& c) const {
    c.assign((size_t)count * rows_total_, 0.0);
    if (sph_h_.empty() || count <= 0) return;
    ensure(sc, count);
    launch_nl_project(L, static_cast<const Sphere*>(spheres_.p), (int)sph_h_.size(), static_cast<const int*>(chunk_sphere_.p),
                      total_chunks_, beta_.f(), x, count, rows_total_, sc.partials.d(), sc.coef.d(), s);
    KS_CUDA(cudaMemcpyAsync(c.data(), sc.coef.p, c.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    KS_CUDA(cudaStreamSynchronize(s));
}

// sums[(v * rows + row) * 4 + {x, y, z, beta}] = h^3 sum over the row's ball of (grad beta, beta) psi_v, chunk
// partials summed in chunk order (Neumaier) on the host
void Ionic::nl_force_sums(const Layout& L, const float* psi, int count, Scratch& sc, cudaStream_t s, std::vector<double>& sums) const {
    sums.assign((size_t)count * rows_total_ * 4, 0.0);
    if (sph_h_.empty() || count <= 0) return;
    ensure(sc, count);
    launch_nl_forces(L, static_cast<const Sphere*>(spheres_.p), static_cast<const int*>(chunk_sphere_.p), total_chunks_, psi, count,
                     rows_total_, sc.partials.d(), s);
    std::vector<double> part((size_t)count * rows_total_ * MAX_CHUNKS * 4);
    KS_CUDA(cudaMemcpyAsync(part.data(), sc.partials.p, part.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    KS_CUDA(cudaStreamSynchronize(s));
    const double dv = L.h * L.h * L.h;
    for (int v = 0; v < count; ++v)
        for (const Sphere& sp : sph_h_)
            for (int r = 0; r < sp.rows; ++r)
                for (int a = 0; a < 4; ++a) {
                    double sum = 0.0, comp = 0.0;
                    for (int ch = 0; ch < sp.chunks; ++ch) {
                        const double x = part[(((size_t)v * rows_total_ + sp.row0 + r) * MAX_CHUNKS + ch) * 4 + a];
                        const double t = sum + x;
                        if (std::fabs(sum) >= std::fabs(x)) comp += (sum - t) + x; else comp += (x - t) + sum;
                        sum = t;
                    }
                    sums[((size_t)v * rows_total_ + sp.row0 + r) * 4 + a] = (sum + comp) * dv;
                }
}

}  // namespace ks
