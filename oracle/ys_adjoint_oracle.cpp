// ys_adjoint_oracle.cpp -- FP64 CPU reference of the differentiable cloth
// rollout: forward substeps and their hand-derived adjoint.
//
// TEST INFRASTRUCTURE ONLY (gradient checks of the CUDA adjoint).
//
// Forward step (SymplecticSystem<METAL>::update for one FastGridCloth,
// physics.metal:146-312, with per-spring stiffness k_s and rest length L_s):
//   f_i  = ext_i + kair v_i + sum_s (k_s (l - L_s) + kd (dv . n)) n
//   v'   = v + (subh f / m) mask
//   for each contact c (n_c, d_c) of vertex i, in (object, triangle) order:
//       if d_c < thickness: { if v'.n_c < 0: v' -= (v'.n_c) n_c;  x += (thickness - d_c) n_c }
//   x'   = x + subh v' mask
// Contacts come from the static obstacle: narrow_pt_tri (bruteforce.metal:41-178)
// on the candidates of a point query with box x +- margin (queryPoints,
// bvh.metal:1322-1412) against triangles whose AABB it overlaps; d_c =
// n_c . (x - t0_c) with n_c fixed by the triangle and the orientation rule.
// The adjoint freezes the active set of the forward pass (which contacts
// exist, which push, which project the velocity), so it is exact for the
// piecewise-smooth map.
//
// Grid springs: 6 families with canonical ids (the enumeration the CUDA path
// uses), gathered per vertex in the stencil order of
// compute_cloth_grid_forces_fast (physics.metal:197-218).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

struct D3 { double x, y, z; };
inline D3 d3(double a, double b, double c) { return D3{a, b, c}; }
inline D3 operator+(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline D3 operator-(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline D3 operator*(D3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) { return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline D3 ld(const std::vector<double>& v, size_t i) { return d3(v[3 * i], v[3 * i + 1], v[3 * i + 2]); }
inline void st(std::vector<double>& v, size_t i, D3 a) { v[3 * i] = a.x; v[3 * i + 1] = a.y; v[3 * i + 2] = a.z; }
inline void add(std::vector<double>& v, size_t i, D3 a) { v[3 * i] += a.x; v[3 * i + 1] += a.y; v[3 * i + 2] += a.z; }

struct Nb { uint32_t j, s; };  // neighbour vertex, spring id

struct Contact { D3 n; double d; D3 t0; };

struct Roll {
    int N = 0;
    size_t V = 0, S = 0;
    std::vector<double> x0, v0, k, L, mass, mask;
    double kd = 0.5, kair = -0.001, subh = 1.0 / 600.0, thickness = 1e-3, margin = 0.015, radius = 0.012;
    D3 g{0, -9.81, 0};
    std::vector<double> ox;           // obstacle vertices
    std::vector<uint32_t> oF;         // obstacle faces
    std::vector<double> obmin, obmax; // per-face AABB
    D3 orootmin, orootmax;
    // static uniform grid over the obstacle's face boxes (candidate search)
    double cell = 1.0;
    std::unordered_map<uint64_t, std::vector<uint32_t>> grid;
    static uint64_t key(long long x, long long y, long long z) {
        return ((uint64_t)(x + (1 << 20)) & 0x1FFFFF) | (((uint64_t)(y + (1 << 20)) & 0x1FFFFF) << 21) |
               (((uint64_t)(z + (1 << 20)) & 0x1FFFFF) << 42);
    }
    void build_grid() {
        const size_t nf = oF.size() / 3;
        double ext = 1e-6;
        for (size_t f = 0; f < nf; ++f)
            for (int a = 0; a < 3; ++a) ext = std::max(ext, obmax[3 * f + a] - obmin[3 * f + a]);
        cell = ext;
        for (size_t f = 0; f < nf; ++f) {
            long long lo[3], hi[3];
            for (int a = 0; a < 3; ++a) {
                lo[a] = (long long)std::floor(obmin[3 * f + a] / cell);
                hi[a] = (long long)std::floor(obmax[3 * f + a] / cell);
            }
            for (long long z = lo[2]; z <= hi[2]; ++z)
                for (long long y = lo[1]; y <= hi[1]; ++y)
                    for (long long x = lo[0]; x <= hi[0]; ++x) grid[key(x, y, z)].push_back((uint32_t)f);
        }
    }
    // per-vertex springs in stencil order
    std::vector<std::vector<Nb>> nbs;
    // trajectory (for the backward pass)
    std::vector<std::vector<double>> xs, vs;
    std::vector<std::vector<std::vector<Contact>>> cs;  // contacts per step per vertex

    void springs() {
        nbs.assign(V, {});
        const uint32_t n = (uint32_t)N;
        const size_t bSY = (size_t)n * (n - 1), bHA = bSY + (size_t)(n - 1) * n, bHB = bHA + (size_t)(n - 1) * (n - 1),
                     bBX = bHB + (size_t)(n - 1) * (n - 1), bBY = bBX + (size_t)n * (n - 2);
        S = bBY + (size_t)(n - 2) * n;
        for (uint32_t r = 0; r < n; ++r)
            for (uint32_t c = 0; c < n; ++c) {
                auto& v = nbs[r * n + c];
                auto id = [&](uint32_t rr, uint32_t cc) { return rr * n + cc; };
                if (c > 0) v.push_back({id(r, c - 1), (uint32_t)(r * (n - 1) + c - 1)});
                if (c < n - 1) v.push_back({id(r, c + 1), (uint32_t)(r * (n - 1) + c)});
                if (r > 0) v.push_back({id(r - 1, c), (uint32_t)(bSY + (r - 1) * n + c)});
                if (r < n - 1) v.push_back({id(r + 1, c), (uint32_t)(bSY + r * n + c)});
                if (c > 0 && r > 0) v.push_back({id(r - 1, c - 1), (uint32_t)(bHA + (r - 1) * (n - 1) + c - 1)});
                if (c < n - 1 && r > 0) v.push_back({id(r - 1, c + 1), (uint32_t)(bHB + (r - 1) * (n - 1) + c)});
                if (c > 0 && r < n - 1) v.push_back({id(r + 1, c - 1), (uint32_t)(bHB + r * (n - 1) + c - 1)});
                if (c < n - 1 && r < n - 1) v.push_back({id(r + 1, c + 1), (uint32_t)(bHA + r * (n - 1) + c)});
                if (c > 1) v.push_back({id(r, c - 2), (uint32_t)(bBX + r * (n - 2) + c - 2)});
                if (c < n - 2) v.push_back({id(r, c + 2), (uint32_t)(bBX + r * (n - 2) + c)});
                if (r > 1) v.push_back({id(r - 2, c), (uint32_t)(bBY + (r - 2) * n + c)});
                if (r < n - 2) v.push_back({id(r + 2, c), (uint32_t)(bBY + r * n + c)});
            }
    }

    // narrow_pt_tri in double; returns contact or false
    bool narrow(D3 qc, D3 qp, uint32_t f, Contact& out) const {
        D3 t0 = ld(ox, oF[3 * f]), t1 = ld(ox, oF[3 * f + 1]), t2 = ld(ox, oF[3 * f + 2]);
        D3 e0 = t1 - t0, e1 = t2 - t0;
        D3 n = cross(e0, e1);
        double nl2 = dot(n, n);
        if (nl2 < 1e-12) return false;
        n = n * (1.0 / std::sqrt(nl2));
        double dp = dot(n, qp - t0), dc = dot(n, qc - t0);
        double dref = (dp != 0.0) ? dp : dc;
        if (dref < 0.0) { n = n * -1.0; dp = -dp; dc = -dc; }
        bool crossed = dc < 0.0, inm = dc < radius + margin;
        if (!crossed && !inm) return false;
        D3 cp = (crossed && dp > 0.0) ? qp + (qc - qp) * (dp / (dp - dc)) : qc;
        D3 pc = cp - t0;
        D3 inplane = pc - n * dot(n, pc);
        double d00 = dot(e0, e0), d01 = dot(e0, e1), d11 = dot(e1, e1), d20 = dot(inplane, e0), d21 = dot(inplane, e1);
        double den = d00 * d11 - d01 * d01;
        if (std::fabs(den) < 1e-12) return false;
        double b = (d11 * d20 - d01 * d21) / den, c = (d00 * d21 - d01 * d20) / den, a = 1.0 - b - c;
        if (!(a >= 0.0 && b >= 0.0 && c >= 0.0)) return false;
        out.n = n; out.d = dc; out.t0 = t0;
        return true;
    }

    void contacts(const std::vector<double>& x, const std::vector<double>& xp, const std::vector<double>& v,
                  std::vector<std::vector<Contact>>& out) const {
        out.assign(V, {});
        // root cull: swept cloth box vs obstacle root box
        D3 lo = ld(x, 0), hi = lo;
        for (size_t i = 0; i < V; ++i) {
            D3 p = ld(x, i), s = p + ld(v, i) * subh;
            lo = d3(std::fmin(lo.x, std::fmin(p.x, s.x)), std::fmin(lo.y, std::fmin(p.y, s.y)), std::fmin(lo.z, std::fmin(p.z, s.z)));
            hi = d3(std::fmax(hi.x, std::fmax(p.x, s.x)), std::fmax(hi.y, std::fmax(p.y, s.y)), std::fmax(hi.z, std::fmax(p.z, s.z)));
        }
        if (hi.x < orootmin.x || lo.x > orootmax.x || hi.y < orootmin.y || lo.y > orootmax.y || hi.z < orootmin.z ||
            lo.z > orootmax.z)
            return;
#pragma omp parallel for schedule(dynamic, 64)
        for (long long il = 0; il < (long long)V; ++il) {
            size_t i = (size_t)il;
            D3 p = ld(x, i), pp = ld(xp, i);
            D3 qmn = p - d3(margin, margin, margin), qmx = p + d3(margin, margin, margin);
            std::vector<uint32_t> cand;
            const double qa[3] = {qmn.x, qmn.y, qmn.z}, qb[3] = {qmx.x, qmx.y, qmx.z};
            long long lo[3], hi[3];
            for (int a = 0; a < 3; ++a) { lo[a] = (long long)std::floor(qa[a] / cell); hi[a] = (long long)std::floor(qb[a] / cell); }
            for (long long z = lo[2]; z <= hi[2]; ++z)
                for (long long y = lo[1]; y <= hi[1]; ++y)
                    for (long long xx = lo[0]; xx <= hi[0]; ++xx) {
                        auto it = grid.find(key(xx, y, z));
                        if (it != grid.end()) cand.insert(cand.end(), it->second.begin(), it->second.end());
                    }
            std::sort(cand.begin(), cand.end());
            cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
            for (uint32_t f : cand) {
                if (qmx.x < obmin[3 * f] || qmn.x > obmax[3 * f] || qmx.y < obmin[3 * f + 1] || qmn.y > obmax[3 * f + 1] ||
                    qmx.z < obmin[3 * f + 2] || qmn.z > obmax[3 * f + 2])
                    continue;
                Contact c;
                if (narrow(p, pp, (uint32_t)f, c)) out[i].push_back(c);  // ascending triangle order
            }
        }
    }

    D3 force(const std::vector<double>& x, const std::vector<double>& v, size_t i) const {
        D3 p = ld(x, i), w = ld(v, i);
        D3 f = g * mass[i] + w * kair;
        for (const Nb& e : nbs[i]) {
            D3 dx = ld(x, e.j) - p, dv = ld(v, e.j) - w;
            double l = std::sqrt(dot(dx, dx));
            if (l < 1e-7) continue;
            D3 nd = dx * (1.0 / l);
            f = f + nd * (k[e.s] * (l - L[e.s]) + kd * dot(dv, nd));
        }
        return f;
    }

    void forward(int T, bool keep) {
        std::vector<double> x = x0, v = v0, xp = x0;
        if (keep) { xs.assign(1, x); vs.assign(1, v); cs.clear(); }
        for (int t = 0; t < T; ++t) {
            std::vector<std::vector<Contact>> C;
            contacts(x, xp, v, C);
            std::vector<double> xn(3 * V), vn(3 * V);
#pragma omp parallel for schedule(static)
            for (long long il = 0; il < (long long)V; ++il) {
                size_t i = (size_t)il;
                D3 f = force(x, v, i);
                D3 vel = ld(v, i) + f * (subh / mass[i] * mask[i]);
                D3 pos = ld(x, i);
                for (const Contact& c : C[i]) {
                    if (c.d < thickness) {
                        double vn_ = dot(vel, c.n);
                        if (vn_ < 0.0) vel = vel - c.n * vn_;
                        pos = pos + c.n * (thickness - c.d);
                    }
                }
                pos = pos + vel * (subh * mask[i]);
                st(xn, i, pos);
                st(vn, i, vel);
            }
            xp = x;
            x.swap(xn);
            v.swap(vn);
            if (keep) { xs.push_back(x); vs.push_back(v); cs.push_back(std::move(C)); }
        }
        if (!keep) { xs.assign(1, x); vs.assign(1, v); }
    }

    // reverse pass; ax, av = dL/dx_T, dL/dv_T on entry
    void backward(int T, std::vector<double> ax, std::vector<double> av, std::vector<double>& gk,
                  std::vector<double>& gL, std::vector<double>& gv0, std::vector<double>& gx0) {
        gk.assign(S, 0.0); gL.assign(S, 0.0);
        for (int t = T - 1; t >= 0; --t) {
            const std::vector<double>& x = xs[t];
            const std::vector<double>& v = vs[t];
            const auto& C = cs[t];
            std::vector<double> fbar(3 * V), xbar(3 * V), vbar(3 * V);
            // per-vertex: x' = P(x) + subh mask v'',  v'' = Q(v'),  v' = v + subh/m mask f
#pragma omp parallel for schedule(static)
            for (long long il = 0; il < (long long)V; ++il) {
                size_t i = (size_t)il;
                D3 f = force(x, v, i);
                D3 vel = ld(v, i) + f * (subh / mass[i] * mask[i]);
                // replay the projections to freeze the active set
                std::vector<char> proj(C[i].size(), 0);
                for (size_t c = 0; c < C[i].size(); ++c)
                    if (C[i][c].d < thickness) {
                        double vn_ = dot(vel, C[i][c].n);
                        if (vn_ < 0.0) { vel = vel - C[i][c].n * vn_; proj[c] = 1; }
                    }
                D3 axi = ld(ax, i);
                D3 vb = ld(av, i) + axi * (subh * mask[i]);       // dL/dv''
                for (size_t c = C[i].size(); c-- > 0;)               // Q^T, reverse order
                    if (proj[c]) vb = vb - C[i][c].n * dot(C[i][c].n, vb);
                D3 xb = axi;                                          // P^T
                for (const Contact& c : C[i])
                    if (c.d < thickness) xb = xb - c.n * dot(c.n, axi);
                st(xbar, i, xb);
                st(vbar, i, vb);                                      // through v' = v + ...
                st(fbar, i, vb * (subh / mass[i] * mask[i]));
            }
            // springs + air drag (gather per vertex, spring params by owner)
            std::vector<double> xb2 = xbar, vb2 = vbar;
#pragma omp parallel for schedule(static)
            for (long long il = 0; il < (long long)V; ++il) {
                size_t i = (size_t)il;
                D3 p = ld(x, i), w = ld(v, i);
                D3 fi = ld(fbar, i);
                D3 dxb{0, 0, 0}, dvb{0, 0, 0};
                for (const Nb& e : nbs[i]) {
                    D3 dx = ld(x, e.j) - p, dv = ld(v, e.j) - w;
                    double l = std::sqrt(dot(dx, dx));
                    if (l < 1e-7) continue;
                    D3 nd = dx * (1.0 / l);
                    double a = k[e.s] * (l - L[e.s]) + kd * dot(dv, nd);
                    // F_s acts +F on i (from i's gather) and -F on j:  g = fbar_i - fbar_j
                    D3 gdir = fi - ld(fbar, e.j);
                    double ng = dot(nd, gdir);
                    // dF/d(dx)^T g = (k n + kd (I - nn^T) dv / l)(n.g) + a/l (I - nn^T) g
                    D3 dvp = dv - nd * dot(nd, dv), gp = gdir - nd * ng;
                    D3 ddx = nd * (k[e.s] * ng) + dvp * (kd * ng / l) + gp * (a / l);
                    D3 ddv = nd * (kd * ng);
                    dxb = dxb - ddx;   // dx = x_j - x_i
                    dvb = dvb - ddv;
                    if (i < e.j) { gk[e.s] += (l - L[e.s]) * ng; gL[e.s] += -k[e.s] * ng; }
                }
                add(xb2, i, dxb);
                add(vb2, i, dvb + fi * kair);
            }
            ax.swap(xb2);
            av.swap(vb2);
        }
        gv0 = av;
        gx0 = ax;
    }
};

}  // namespace

extern "C" {

// ip: N, obstacle vertices, obstacle faces.  dp: kd, kair, subh, thickness,
// margin, radius, gx, gy, gz.
void* yso_roll_new(const int* ip, const double* dp, const double* x0, const double* v0, const double* mass,
                   const double* mask, const double* ox, const uint32_t* oF) {
    Roll* R = new Roll();
    R->N = ip[0];
    R->V = (size_t)R->N * R->N;
    R->kd = dp[0]; R->kair = dp[1]; R->subh = dp[2]; R->thickness = dp[3]; R->margin = dp[4]; R->radius = dp[5];
    R->g = d3(dp[6], dp[7], dp[8]);
    R->x0.assign(x0, x0 + 3 * R->V);
    R->v0.assign(v0, v0 + 3 * R->V);
    R->mass.assign(mass, mass + R->V);
    R->mask.assign(mask, mask + R->V);
    R->ox.assign(ox, ox + 3 * (size_t)ip[1]);
    R->oF.assign(oF, oF + 3 * (size_t)ip[2]);
    const size_t nf = (size_t)ip[2];
    R->obmin.resize(3 * nf); R->obmax.resize(3 * nf);
    R->orootmin = d3(1e300, 1e300, 1e300); R->orootmax = d3(-1e300, -1e300, -1e300);
    for (size_t f = 0; f < nf; ++f)
        for (int a = 0; a < 3; ++a) {
            double p0 = R->ox[3 * R->oF[3 * f] + a], p1 = R->ox[3 * R->oF[3 * f + 1] + a], p2 = R->ox[3 * R->oF[3 * f + 2] + a];
            R->obmin[3 * f + a] = std::fmin(p0, std::fmin(p1, p2));
            R->obmax[3 * f + a] = std::fmax(p0, std::fmax(p1, p2));
        }
    for (size_t f = 0; f < nf; ++f) {
        R->orootmin = d3(std::fmin(R->orootmin.x, R->obmin[3 * f]), std::fmin(R->orootmin.y, R->obmin[3 * f + 1]), std::fmin(R->orootmin.z, R->obmin[3 * f + 2]));
        R->orootmax = d3(std::fmax(R->orootmax.x, R->obmax[3 * f]), std::fmax(R->orootmax.y, R->obmax[3 * f + 1]), std::fmax(R->orootmax.z, R->obmax[3 * f + 2]));
    }
    R->build_grid();
    R->springs();
    R->k.assign(R->S, 0.0);
    R->L.assign(R->S, 0.0);
    return R;
}
void yso_roll_free(void* h) { delete (Roll*)h; }
uint64_t yso_roll_num_springs(void* h) { return ((Roll*)h)->S; }
void yso_roll_set(void* h, const double* k, const double* L, const double* v0) {
    Roll* R = (Roll*)h;
    if (k) R->k.assign(k, k + R->S);
    if (L) R->L.assign(L, L + R->S);
    if (v0) R->v0.assign(v0, v0 + 3 * R->V);
}
// forward T steps; x_out receives x_T; returns the number of contacts seen
uint64_t yso_roll_forward(void* h, int T, int keep, double* x_out) {
    Roll* R = (Roll*)h;
    R->forward(T, keep != 0);
    if (x_out) std::memcpy(x_out, R->xs.back().data(), 8 * 3 * R->V);
    uint64_t n = 0;
    for (auto& step : R->cs) for (auto& c : step) n += c.size();
    return n;
}
void yso_roll_backward(void* h, int T, const double* ax, double* gk, double* gL, double* gv0) {
    Roll* R = (Roll*)h;
    std::vector<double> a(ax, ax + 3 * R->V), b(3 * R->V, 0.0), k_, L_, v_, x_;
    R->backward(T, a, b, k_, L_, v_, x_);
    std::memcpy(gk, k_.data(), 8 * R->S);
    std::memcpy(gL, L_.data(), 8 * R->S);
    std::memcpy(gv0, v_.data(), 8 * 3 * R->V);
}

}  // extern "C"
