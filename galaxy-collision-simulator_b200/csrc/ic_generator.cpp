// ic_generator.cpp - seeded two-galaxy initial conditions.
//
// Components follow the reference's generator (generator.cpp:3-196): a
// Miyamoto-Nagai disc drawn by rejection against the MN density
// (generator.cpp:31-37), Hernquist bulge and dark-matter halo drawn by the
// Hernquist inverse CDF (generator.cpp:76-78,136-138), colours and types of
// its palette (generator.cpp:150-152,175-176,199-207), particles ordered
// halo, disc, bulge per galaxy.  Parameters, truncations, velocities and the
// orbit are the recipe's, not the reference's hard-coded ones:
//   * disc positions: rejection sampling with a separable envelope
//     (R ~ R/(R^2+c^2)^{3/2}, z ~ (z^2+b^2)^{-3/2}, c = a+b), which bounds
//     the MN density everywhere inside the truncation box;
//   * disc velocities: circular speed of the combined potential in the
//     plane (MN disc + two truncated Hernquist spheres) plus isotropic
//     Gaussian noise of 0.1 v_c per axis;
//   * bulge/halo velocities: isotropic Gaussian with sigma^2(r) from the
//     isotropic Jeans equation in the combined spherically averaged mass
//     profile, integrated numerically on a log grid;
//   * every draw comes from a counter-based stream keyed by (seed, galaxy,
//     component, chunk), so output is identical for any thread count.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/gcs.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// xoshiro256** (Blackman & Vigna 2018).
struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (auto& w : s) w = splitmix64(x);
    }
    static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
    double normal() {  // Box-Muller, one value per call
        double u1 = uniform();
        while (u1 <= 0.0) u1 = uniform();
        const double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
    }
    void direction(double& x, double& y, double& z) {
        const double c = 2.0 * uniform() - 1.0;
        const double s = std::sqrt(std::max(0.0, 1.0 - c * c));
        const double ph = 2.0 * kPi * uniform();
        x = s * std::cos(ph);
        y = s * std::sin(ph);
        z = c;
    }
};

uint64_t stream_key(uint64_t seed, int galaxy, int comp, int64_t chunk) {
    uint64_t x = seed ^ 0x5DEECE66Dull;
    uint64_t k = splitmix64(x);
    k ^= (uint64_t)(galaxy * 8 + comp) * 0xD1B54A32D192ED03ull;
    k ^= (uint64_t)chunk * 0x9E3779B97F4A7C15ull;
    uint64_t y = k;
    return splitmix64(y);
}

// Fraction of a Hernquist sphere's mass inside r.
double hern_frac(double r, double a) { return (r * r) / ((r + a) * (r + a)); }

// Mass of one galaxy inside radius r (spherical average), truncations honoured.
struct MassModel {
    const gcs_galaxy_spec* g;
    double enclosed(double r) const {
        double m = 0.0;
        // disc: Plummer-like spherical average of the MN profile, capped at its mass
        const double c = (double)g->disc_a + g->disc_b;
        m += g->disc_mass * std::pow(r * r / (r * r + c * c), 1.5);
        const double rb = std::min(r, (double)g->bulge_rmax);
        m += g->bulge_mass * hern_frac(rb, g->bulge_a) / hern_frac(g->bulge_rmax, g->bulge_a);
        const double rh = std::min(r, (double)g->halo_rmax);
        m += g->halo_mass * hern_frac(rh, g->halo_a) / hern_frac(g->halo_rmax, g->halo_a);
        return m;
    }
    // In-plane circular speed squared at cylindrical radius R (z = 0).
    double vc2(double R, double G) const {
        const double c = (double)g->disc_a + g->disc_b;
        double v2 = G * g->disc_mass * R * R / std::pow(R * R + c * c, 1.5);
        const double rb = std::min(R, (double)g->bulge_rmax);
        v2 += G * g->bulge_mass * hern_frac(rb, g->bulge_a) / hern_frac(g->bulge_rmax, g->bulge_a) / R;
        const double rh = std::min(R, (double)g->halo_rmax);
        v2 += G * g->halo_mass * hern_frac(rh, g->halo_a) / hern_frac(g->halo_rmax, g->halo_a) / R;
        return v2;
    }
};

// sigma^2(r) of an isotropic truncated Hernquist component in the galaxy's
// mass profile: sigma^2 = (1/rho) * int_r^rt rho(r') G M(r') / r'^2 dr'.
struct JeansTable {
    std::vector<double> lr, s2;
    double lo = 0, hi = 0, step = 0;
    void build(const MassModel& mm, double a, double rt, double G) {
        const int n = 512;
        lo = std::log(a * 1e-4);
        hi = std::log(rt);
        step = (hi - lo) / (n - 1);
        lr.resize(n);
        s2.assign(n, 0.0);
        auto rho = [a](double r) { return 1.0 / (r * std::pow(r + a, 3)); };
        std::vector<double> integrand(n);
        for (int i = 0; i < n; ++i) {
            lr[i] = lo + step * i;
            const double r = std::exp(lr[i]);
            // d r = r d ln r
            integrand[i] = rho(r) * G * mm.enclosed(r) / (r * r) * r;
        }
        double acc = 0.0;
        s2[n - 1] = 0.0;
        for (int i = n - 2; i >= 0; --i) {
            acc += 0.5 * (integrand[i] + integrand[i + 1]) * step;
            s2[i] = acc / rho(std::exp(lr[i]));
        }
    }
    double at(double r) const {
        const double x = (std::log(std::max(r, std::exp(lo))) - lo) / step;
        int i = (int)x;
        if (i < 0) return s2.front();
        if (i >= (int)s2.size() - 1) return s2.back();
        const double f = x - i;
        return s2[i] * (1 - f) + s2[i + 1] * f;
    }
};

struct Palette {
    uint8_t disc[3], bulge[3];
};

void place(Star& s, const gcs_galaxy_spec& g, double x, double y, double z, double vx, double vy,
           double vz) {
    const double inc = g.incline_deg * kPi / 180.0;
    const double c = std::cos(inc), sn = std::sin(inc);
    const double y2 = y * c - z * sn, z2 = y * sn + z * c;
    const double vy2 = vy * c - vz * sn, vz2 = vy * sn + vz * c;
    s.x = (float)(x + g.pos[0]);
    s.y = (float)(y2 + g.pos[1]);
    s.z = (float)(z2 + g.pos[2]);
    s.vx = (float)(vx + g.vel[0]);
    s.vy = (float)(vy2 + g.vel[1]);
    s.vz = (float)(vz2 + g.vel[2]);
}

constexpr int64_t kChunk = 16384;

void gen_disc_chunk(const gcs_galaxy_spec& g, double G, double disp, const MassModel& mm,
                    const Palette& pal, Star* out, int64_t n, Rng rng) {
    const double a = g.disc_a, b = g.disc_b, Rmax = g.disc_rmax, zmax = g.disc_zmax;
    const double c = a + b;
    const double zeta_max = std::sqrt(zmax * zmax + b * b);
    const double kbound = a + 3.0 * zeta_max;
    const double wr = 1.0 / c - 1.0 / std::sqrt(Rmax * Rmax + c * c);
    const double vmax = zmax / std::sqrt(zmax * zmax + b * b);
    const double mass = (double)g.disc_mass / (double)g.n_disc;
    for (int64_t i = 0; i < n; ++i) {
        double R, z;
        for (;;) {
            const double w = 1.0 / c - rng.uniform() * wr;
            R = std::sqrt(std::max(0.0, 1.0 / (w * w) - c * c));
            const double v = (2.0 * rng.uniform() - 1.0) * vmax;
            z = b * v / std::sqrt(1.0 - v * v);
            const double zeta = std::sqrt(z * z + b * b);
            const double az = a + zeta;
            const double num = a * R * R + (a + 3.0 * zeta) * az * az;
            const double q2 = R * R + az * az;
            const double ratio = num / std::pow(q2, 2.5) * std::pow(R * R + c * c, 1.5) / kbound;
            if (rng.uniform() < ratio && R > 0.0) break;
        }
        const double ph = 2.0 * kPi * rng.uniform();
        const double x = R * std::cos(ph), y = R * std::sin(ph);
        const double vc = std::sqrt(mm.vc2(R, G));
        const double vx = -vc * y / R + disp * vc * rng.normal();
        const double vy = vc * x / R + disp * vc * rng.normal();
        const double vz = disp * vc * rng.normal();
        Star& s = out[i];
        place(s, g, x, y, z, vx, vy, vz);
        s.mass = (float)mass;
        s.type = g.type;
        s.r = pal.disc[0];
        s.g = pal.disc[1];
        s.b = pal.disc[2];
    }
}

void gen_sphere_chunk(const gcs_galaxy_spec& g, double M, double a, double rt, int64_t count,
                      const JeansTable& jt, uint8_t type, const uint8_t rgb[3], Star* out,
                      int64_t n, Rng rng) {
    const double ft = hern_frac(rt, a);
    const double mass = M / (double)count;
    for (int64_t i = 0; i < n; ++i) {
        const double u = rng.uniform() * ft;
        const double su = std::sqrt(u);
        const double r = a * su / (1.0 - su);
        double dx, dy, dz;
        rng.direction(dx, dy, dz);
        const double sig = std::sqrt(std::max(0.0, jt.at(r)));
        Star& s = out[i];
        place(s, g, r * dx, r * dy, r * dz, sig * rng.normal(), sig * rng.normal(), sig * rng.normal());
        s.mass = (float)mass;
        s.type = type;
        s.r = rgb[0];
        s.g = rgb[1];
        s.b = rgb[2];
    }
}

struct Task {
    int galaxy, comp;
    int64_t chunk, first, n;
};

void fill_galaxy_common(gcs_galaxy_spec& g) {
    g.disc_mass = 1.0f;
    g.disc_a = 3.0f;
    g.disc_b = 0.3f;
    g.disc_rmax = 15.0f;
    g.disc_zmax = 3.0f;
    g.bulge_mass = 0.33f;
    g.bulge_a = 0.5f;
    g.bulge_rmax = 5.0f;
    g.halo_mass = 5.8f;
    g.halo_a = 10.0f;
    g.halo_rmax = 30.0f;
    g.incline_deg = 0.0f;
    for (int k = 0; k < 3; ++k) g.pos[k] = g.vel[k] = 0.0f;
}

void split_counts(int64_t n_gal, int64_t& disc, int64_t& bulge, int64_t& halo) {
    disc = (int64_t)std::llround((double)n_gal * 384000.0 / 524288.0);
    bulge = (int64_t)std::llround((double)n_gal * 96000.0 / 524288.0);
    halo = n_gal - disc - bulge;
    if (halo < 0) {
        halo = 0;
        bulge = n_gal - disc;
    }
}

}  // namespace

extern "C" {

int gcs_collision_spec_equal(gcs_collision_spec* spec, int64_t n_disc, int64_t n_bulge,
                             int64_t n_halo, uint64_t seed) {
    if (!spec || n_disc < 0 || n_bulge < 0 || n_halo < 0) return GCS_ERR_ARG;
    memset(spec, 0, sizeof *spec);
    for (int k = 0; k < 2; ++k) {
        gcs_galaxy_spec& g = spec->galaxy[k];
        fill_galaxy_common(g);
        g.n_disc = n_disc;
        g.n_bulge = n_bulge;
        g.n_halo = n_halo;
    }
    spec->galaxy[0].pos[0] = -20.0f;
    spec->galaxy[0].pos[1] = -5.0f;
    spec->galaxy[0].vel[0] = 0.4f;
    spec->galaxy[0].type = 0;
    spec->galaxy[1].pos[0] = 20.0f;
    spec->galaxy[1].pos[1] = 5.0f;
    spec->galaxy[1].vel[0] = -0.4f;
    spec->galaxy[1].incline_deg = 30.0f;
    spec->galaxy[1].type = 2;
    spec->seed = seed;
    spec->G = 1.0f;
    spec->disc_dispersion = 0.1f;
    return GCS_OK;
}

int gcs_collision_spec_pair(gcs_collision_spec* spec, int64_t n_total, float q, float impact,
                            float rel_speed, float incline_deg, uint64_t seed) {
    if (!spec || n_total < 2 || !(q > 0.0f && q <= 1.0f)) return GCS_ERR_ARG;
    memset(spec, 0, sizeof *spec);
    const double mq = q;
    const double ls = std::cbrt(mq);
    const int64_t n_a = std::max<int64_t>(1, (int64_t)std::llround((double)n_total * mq / (1.0 + mq)));
    const int64_t n_b = n_total - n_a;
    gcs_galaxy_spec& A = spec->galaxy[0];
    gcs_galaxy_spec& B = spec->galaxy[1];
    fill_galaxy_common(A);
    fill_galaxy_common(B);
    A.disc_mass *= (float)mq;
    A.bulge_mass *= (float)mq;
    A.halo_mass *= (float)mq;
    A.disc_a *= (float)ls;
    A.disc_b *= (float)ls;
    A.disc_rmax *= (float)ls;
    A.disc_zmax *= (float)ls;
    A.bulge_a *= (float)ls;
    A.bulge_rmax *= (float)ls;
    A.halo_a *= (float)ls;
    A.halo_rmax *= (float)ls;
    split_counts(n_a, A.n_disc, A.n_bulge, A.n_halo);
    split_counts(n_b, B.n_disc, B.n_bulge, B.n_halo);
    const double fa = 1.0 / (1.0 + mq), fb = mq / (1.0 + mq);  // M_B/M, M_A/M
    A.pos[0] = (float)(-40.0 * fa);
    A.pos[1] = (float)(-impact * fa);
    A.vel[0] = (float)(rel_speed * fa);
    B.pos[0] = (float)(40.0 * fb);
    B.pos[1] = (float)(impact * fb);
    B.vel[0] = (float)(-rel_speed * fb);
    A.type = 0;
    B.type = 2;
    B.incline_deg = incline_deg;
    spec->seed = seed;
    spec->G = 1.0f;
    spec->disc_dispersion = 0.1f;
    return GCS_OK;
}

int64_t gcs_collision_count(const gcs_collision_spec* spec) {
    if (!spec) return 0;
    int64_t n = 0;
    for (int k = 0; k < 2; ++k)
        n += spec->galaxy[k].n_disc + spec->galaxy[k].n_bulge + spec->galaxy[k].n_halo;
    return n;
}

int gcs_generate_collision(const gcs_collision_spec* spec, Star* out, int64_t n) {
    if (!spec || !out || n != gcs_collision_count(spec)) return GCS_ERR_ARG;
    const double G = spec->G > 0 ? spec->G : 1.0;
    static const Palette pal[2] = {{{255, 100, 50}, {255, 255, 150}}, {{50, 100, 255}, {200, 255, 255}}};
    static const uint8_t black[3] = {0, 0, 0};
    MassModel mm[2] = {{&spec->galaxy[0]}, {&spec->galaxy[1]}};
    JeansTable jb[2], jh[2];
    for (int k = 0; k < 2; ++k) {
        const gcs_galaxy_spec& g = spec->galaxy[k];
        if (g.n_bulge > 0) jb[k].build(mm[k], g.bulge_a, g.bulge_rmax, G);
        if (g.n_halo > 0) jh[k].build(mm[k], g.halo_a, g.halo_rmax, G);
    }
    std::vector<Task> tasks;
    int64_t first = 0;
    for (int k = 0; k < 2; ++k) {
        const gcs_galaxy_spec& g = spec->galaxy[k];
        const int64_t counts[3] = {g.n_halo, g.n_disc, g.n_bulge};  // reference order: DM, disc, bulge
        for (int comp = 0; comp < 3; ++comp) {
            for (int64_t c0 = 0, ch = 0; c0 < counts[comp]; c0 += kChunk, ++ch)
                tasks.push_back({k, comp, ch, first + c0, std::min(kChunk, counts[comp] - c0)});
            first += counts[comp];
        }
    }
    auto run = [&](const Task& t) {
        const gcs_galaxy_spec& g = spec->galaxy[t.galaxy];
        const Palette& p = pal[g.type == 2 ? 1 : 0];
        Rng rng(stream_key(spec->seed, t.galaxy, t.comp, t.chunk));
        if (t.comp == 0)
            gen_sphere_chunk(g, g.halo_mass, g.halo_a, g.halo_rmax, g.n_halo, jh[t.galaxy], 1, black,
                             out + t.first, t.n, rng);
        else if (t.comp == 1)
            gen_disc_chunk(g, G, spec->disc_dispersion, mm[t.galaxy], p, out + t.first, t.n, rng);
        else
            gen_sphere_chunk(g, g.bulge_mass, g.bulge_a, g.bulge_rmax, g.n_bulge, jb[t.galaxy], g.type,
                             p.bulge, out + t.first, t.n, rng);
    };
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (nt > 32) nt = 32;
    std::vector<std::thread> pool;
    std::atomic_size_t next{0};
    for (unsigned w = 0; w < nt; ++w)
        pool.emplace_back([&]() {
            for (;;) {
                const size_t i = next.fetch_add(1);
                if (i >= tasks.size()) break;
                run(tasks[i]);
            }
        });
    for (auto& th : pool) th.join();
    return GCS_OK;
}

}  // extern "C"
