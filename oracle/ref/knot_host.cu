// knot_host.cu -- TEST INFRASTRUCTURE ONLY.
//
// Host-side driver around the reference's own deterministic packer source,
// cuda/braid_knot.cu, which is #included unmodified from the reference tree
// (its main() is renamed away).  It calls the reference's rng_seed /
// propose / torus_wrap / torus_delta on the CPU and restates the two lambdas
// of braid_knot.cu's main that cannot be called from outside:
//   eval_cand      braid_knot.cu:346-358
//   collides_host  braid_knot.cu:359-372
// The admission loop is braid_knot.cu:433-462 (index order, each survivor
// re-checked against every earlier admission), run sequentially, or as a
// threaded batch prefilter + in-order recheck (--threads N) -- the same
// decisions either way.
//
// Output formats follow braid_knot's --dump file (braid_knot.cu:386-399):
//   "species,attempt" then per axis "a2" and nw x "b,a,f", %.17g.
//
// Modes:
//   --mode stream --first I --count N   candidate parameters for idx in [I, I+N)
//   --mode pack   --attempts A          accepted set, plus "done:" on stderr
#define main braid_knot_reference_main
#include REF_KNOT_SRC
#undef main

#include <chrono>
#include <thread>

namespace {

struct Run {
    int T = 16, dim = 2, terms = 0, pin = 0, threads = 1;
    uint64_t seed = 1;
    long long attempts = 20000, first = 0, count = 16, round = 65536;
    const char* mode = "pack";
};

struct Model {
    int T, dim, nw, pin;
    uint32_t modmax;
    uint64_t seed;
    double cell;
    std::vector<double> sinbz, cosbz, invsinz;
};

void make_model(const Run& r, Model& m) {
    m.T = r.T;
    m.dim = r.dim;
    m.pin = r.pin;
    m.seed = r.seed;
    m.modmax = (uint32_t)(r.T - 1 > 2 ? r.T - 1 : 2);
    m.nw = (r.terms ? r.terms : r.T) - 1;
    m.cell = 2.0 / r.T;
    const int T = r.T, maxfreq = (int)m.modmax + 1;
    std::vector<double> z(T);
    m.invsinz.resize(T);
    for (int i = 0; i < T; i++) {
        z[i] = (i + 1) * kPi / (T + 1);
        m.invsinz[i] = 1.0 / sin(z[i]);
    }
    m.sinbz.resize((size_t)(maxfreq + 1) * T);
    m.cosbz.resize((size_t)(maxfreq + 1) * T);
    for (int b = 0; b <= maxfreq; b++)
        for (int t = 0; t < T; t++) {
            m.sinbz[(size_t)b * T + t] = sin(b * z[t]);
            m.cosbz[(size_t)b * T + t] = cos(b * z[t]);
        }
}

void gen(const Model& m, uint64_t idx, Cand& c) {
    Rng r;
    rng_seed(r, m.seed ^ (idx * 0x9E3779B97F4A7C15ULL + 0x1234567ULL));
    propose(r, m.modmax, m.nw, m.dim, m.pin, c);
}

// braid_knot.cu:346-358
void eval_cand(const Model& m, const Cand& c, std::vector<double>& out) {
    const int T = m.T;
    out.assign((size_t)m.dim * T, 0.0);
    for (int ax = 0; ax < m.dim; ax++)
        for (int t = 0; t < T; t++) {
            double wig = 0.0;
            for (int j = 0; j < m.nw; j++) {
                const int b = c.b[ax][j];
                wig += c.a[ax][j] * (m.sinbz[(size_t)b * T + t] * cos(c.f[ax][j]) +
                                     m.cosbz[(size_t)b * T + t] * sin(c.f[ax][j]) -
                                     sin(c.f[ax][j]));
            }
            out[(size_t)ax * T + t] = torus_wrap(wig * m.invsinz[t] + c.a2[ax]);
        }
}

// braid_knot.cu:359-372, strands laid out [strand][axis][t]
bool collides(const Model& m, const std::vector<double>& pos, const std::vector<double>& strands,
              long long from, long long to) {
    const int T = m.T, D = m.dim;
    for (int t = 0; t < T; t++)
        for (long long s = from; s < to; s++) {
            bool hit = true;
            for (int ax = 0; ax < D; ax++) {
                const double d = torus_delta(pos[(size_t)ax * T + t] -
                                             strands[((size_t)s * D + ax) * T + t]);
                if (fabs(d) > m.cell) {
                    hit = false;
                    break;
                }
            }
            if (hit)
                return true;
        }
    return false;
}

void print_cand(FILE* f, int species, uint64_t attempt, const Model& m, const Cand& c) {
    fprintf(f, "%d,%llu", species, (unsigned long long)attempt);
    for (int ax = 0; ax < m.dim; ax++) {
        fprintf(f, ",%.17g", c.a2[ax]);
        for (int j = 0; j < m.nw; j++)
            fprintf(f, ",%d,%.17g,%.17g", c.b[ax][j], c.a[ax][j], c.f[ax][j]);
    }
    fprintf(f, "\n");
}

}  // namespace

int main(int argc, char** argv) {
    Run r;
    for (int i = 1; i < argc; i++) {
        const char* a = argv[i];
        auto nxt = [&]() { return argv[++i]; };
        if (!strcmp(a, "-t"))
            r.T = atoi(nxt());
        else if (!strcmp(a, "--dim"))
            r.dim = atoi(nxt());
        else if (!strcmp(a, "--terms"))
            r.terms = atoi(nxt());
        else if (!strcmp(a, "--pin-sin1"))
            r.pin = 1;
        else if (!strcmp(a, "--seed"))
            r.seed = strtoull(nxt(), 0, 10);
        else if (!strcmp(a, "--attempts"))
            r.attempts = (long long)atof(nxt());
        else if (!strcmp(a, "--first"))
            r.first = atoll(nxt());
        else if (!strcmp(a, "--count"))
            r.count = atoll(nxt());
        else if (!strcmp(a, "--threads"))
            r.threads = atoi(nxt());
        else if (!strcmp(a, "--round"))
            r.round = atoll(nxt());
        else if (!strcmp(a, "--mode"))
            r.mode = nxt();
        else {
            fprintf(stderr, "unknown flag %s\n", a);
            return 1;
        }
    }
    if (r.dim < 1 || r.dim > 3 || r.T < 4 || r.T > 256) {
        fprintf(stderr, "error: dim 1..3, T 4..256\n");
        return 1;
    }
    Model m;
    make_model(r, m);
    if (m.nw < 1 || m.nw > kMaxW || (uint32_t)m.nw > m.modmax) {
        fprintf(stderr, "error: bad terms\n");
        return 1;
    }
    Cand* c = new Cand;
    if (!strcmp(r.mode, "stream")) {
        for (long long k = 0; k < r.count; k++) {
            gen(m, (uint64_t)(r.first + k), *c);
            print_cand(stdout, 0, (uint64_t)(r.first + k) + 1, m, *c);
        }
        delete c;
        return 0;
    }
    // pack
    std::vector<double> strands;  // [strand][axis][t]
    long long n = 0;
    const size_t rowlen = (size_t)m.dim * m.T;
    std::vector<double> pos;
    auto t0 = std::chrono::steady_clock::now();
    long long idx = 0;
    const int nth = r.threads > 1 ? r.threads : 1;
    std::vector<unsigned char> surv;
    while (idx < r.attempts) {
        const long long cnt = std::min(r.round, r.attempts - idx);
        surv.assign((size_t)cnt, 0);
        const long long n0 = n;
        auto work = [&](int tid) {
            Cand* cc = new Cand;
            std::vector<double> p;
            const long long per = (cnt + nth - 1) / nth;
            const long long lo = tid * per, hi = std::min(cnt, lo + per);
            for (long long k = lo; k < hi; k++) {
                gen(m, (uint64_t)(idx + k), *cc);
                eval_cand(m, *cc, p);
                surv[(size_t)k] = !collides(m, p, strands, 0, n0);
            }
            delete cc;
        };
        if (nth == 1) {
            work(0);
        } else {
            std::vector<std::thread> th;
            for (int k = 0; k < nth; k++)
                th.emplace_back(work, k);
            for (auto& x : th)
                x.join();
        }
        for (long long k = 0; k < cnt; k++) {
            if (!surv[(size_t)k])
                continue;
            gen(m, (uint64_t)(idx + k), *c);
            eval_cand(m, *c, pos);
            if (collides(m, pos, strands, n0, n))
                continue;  // collided with an earlier same-round admission
            strands.insert(strands.end(), pos.begin(), pos.begin() + rowlen);
            n++;
            print_cand(stdout, 0, (uint64_t)(idx + k) + 1, m, *c);
        }
        idx += cnt;
    }
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    fprintf(stderr, "done: N=%lld in %lld attempts (%.6f s, %.1f candidates/s, %d threads)\n", n,
            idx, secs, secs > 0 ? (double)idx / secs : 0.0, nth);
    delete c;
    return 0;
}
