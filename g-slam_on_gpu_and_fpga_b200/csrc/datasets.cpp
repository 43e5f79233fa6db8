/*
 * datasets.cpp — gslam-data, the reference's two dataset tools as one native program:
 *
 *   gslam-data citytrees <n_poses> <output> [seed=42]    data/generate_citytrees.py
 *   gslam-data slampp <input> <output> [delta=1.0]       data/convert_slampp.py
 *
 * The output files are byte-identical to those of the reference scripts run with the
 * same arguments under CPython 3 on the same C math library: the random stream is
 * CPython's (MT19937 seeded by init_by_array, 53-bit random(), rejection-sampled
 * randbelow, the Box-Muller gauss with its cached second value), every float is
 * printed in Python's shortest round-trip repr, and every expression keeps the
 * scripts' operation order (sin, cos, atan2, log, pow and fmod are the C library's,
 * which is what CPython's math module and float operators call; this file is built
 * with -fno-builtin so the compiler neither folds pow(x, 2) into x * x nor merges
 * sin and cos).
 *
 * What is not the scripts': the nearest-landmark and visibility searches use a uniform
 * grid of 9 m cells (larger than the 8.5 m sensor range, so no point within range is
 * ever skipped) instead of scanning every landmark for every pose, which makes large
 * logs (10^5 poses and more) take seconds instead of hours. Candidates are visited in
 * the scripts' order (landmark insertion order, poses in sample order), so the counts
 * capped at MAX_OBS_PER_LM and the observation order are unchanged.
 */
#include <algorithm>
#include <array>
#include <cctype>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

namespace {

const double kPi = 3.141592653589793;

/* ---- CPython's random.Random (MT19937, Matsumoto & Nishimura 1998) ---- */
class PyRandom {
  public:
    explicit PyRandom(uint64_t seed) {
        /* random.seed(int): the absolute value split into 32-bit words, low first */
        std::vector<uint32_t> key;
        do {
            key.push_back((uint32_t)(seed & 0xffffffffu));
            seed >>= 32;
        } while (seed);
        init_by_array(key);
    }

    uint32_t genrand() {
        if (idx_ >= kN) twist();
        uint32_t y = mt_[idx_++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        return y;
    }

    /* random(): 53 bits from two draws */
    double random() {
        const uint32_t a = genrand() >> 5, b = genrand() >> 6;
        return ((double)a * 67108864.0 + (double)b) * (1.0 / 9007199254740992.0);
    }

    /* getrandbits(k), 0 <= k <= 32 */
    uint32_t getrandbits(int k) { return k == 0 ? 0u : genrand() >> (32 - k); }

    /* _randbelow(n): k = bit length of n, draw k bits until below n */
    uint32_t randbelow(uint32_t n) {
        int k = 0;
        while (k < 32 && (n >> k)) k++;
        uint32_t r = getrandbits(k);
        while (r >= n) r = getrandbits(k);
        return r;
    }

    int64_t randint(int64_t a, int64_t b) { return a + (int64_t)randbelow((uint32_t)(b - a + 1)); }

    double uniform(double a, double b) { return a + (b - a) * random(); }

    /* gauss(mu, sigma): Box-Muller pair, the sine half kept for the next call */
    double gauss(double mu, double sigma) {
        double z;
        if (has_next_) {
            z = next_;
            has_next_ = false;
        } else {
            const double x2pi = random() * (2.0 * kPi);
            const double g2rad = std::sqrt(-2.0 * std::log(1.0 - random()));
            z = std::cos(x2pi) * g2rad;
            next_ = std::sin(x2pi) * g2rad;
            has_next_ = true;
        }
        return mu + z * sigma;
    }

  private:
    static const int kN = 624, kM = 397;
    uint32_t mt_[kN];
    int idx_ = kN + 1;
    bool has_next_ = false;
    double next_ = 0.0;

    void init_genrand(uint32_t s) {
        mt_[0] = s;
        for (int i = 1; i < kN; i++) mt_[i] = 1812433253u * (mt_[i - 1] ^ (mt_[i - 1] >> 30)) + (uint32_t)i;
        idx_ = kN;
    }

    void init_by_array(const std::vector<uint32_t> &key) {
        init_genrand(19650218u);
        int i = 1;
        size_t j = 0;
        for (int k = std::max<int>(kN, (int)key.size()); k; k--) {
            mt_[i] = (mt_[i] ^ ((mt_[i - 1] ^ (mt_[i - 1] >> 30)) * 1664525u)) + key[j] + (uint32_t)j;
            i++;
            j++;
            if (i >= kN) { mt_[0] = mt_[kN - 1]; i = 1; }
            if (j >= key.size()) j = 0;
        }
        for (int k = kN - 1; k; k--) {
            mt_[i] = (mt_[i] ^ ((mt_[i - 1] ^ (mt_[i - 1] >> 30)) * 1566083941u)) - (uint32_t)i;
            i++;
            if (i >= kN) { mt_[0] = mt_[kN - 1]; i = 1; }
        }
        mt_[0] = 0x80000000u;
    }

    void twist() {
        for (int k = 0; k < kN; k++) {
            const uint32_t y = (mt_[k] & 0x80000000u) | (mt_[(k + 1) % kN] & 0x7fffffffu);
            mt_[k] = mt_[(k + kM) % kN] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        idx_ = 0;
    }
};

/* ---- Python float semantics ---- */

/* a % b for floats: the remainder takes the sign of b */
double py_mod(double a, double b) {
    double m = std::fmod(a, b);
    if (m != 0.0) {
        if ((b < 0) != (m < 0)) m += b;
    } else {
        m = std::copysign(0.0, b);
    }
    return m;
}

/* repr(float): shortest round-trip digits; positional when the decimal exponent is in
 * (-4, 16], else d.ddde+XX with at least two exponent digits; integral values get ".0" */
std::string py_repr(double v) {
    if (std::isnan(v)) return "nan";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    if (v == 0.0) return std::signbit(v) ? "-0.0" : "0.0";
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
    std::string s(buf, r.ptr);
    std::string out;
    if (s[0] == '-') { out = "-"; s = s.substr(1); }
    const size_t epos = s.find('e');
    std::string digits;
    for (size_t i = 0; i < epos; i++)
        if (s[i] != '.') digits += s[i];
    const int exp10 = atoi(s.c_str() + epos + 1);
    const int decpt = exp10 + 1;             /* value = 0.digits x 10^decpt */
    const int nd = (int)digits.size();
    if (decpt <= -4 || decpt > 16) {
        out += digits[0];
        if (nd > 1) { out += '.'; out += digits.substr(1); }
        char eb[16];
        snprintf(eb, sizeof eb, "e%c%02d", exp10 < 0 ? '-' : '+', std::abs(exp10));
        out += eb;
    } else if (decpt <= 0) {
        out += "0.";
        out += std::string((size_t)(-decpt), '0');
        out += digits;
    } else if (decpt >= nd) {
        out += digits;
        out += std::string((size_t)(decpt - nd), '0');
        out += ".0";
    } else {
        out += digits.substr(0, (size_t)decpt);
        out += '.';
        out += digits.substr((size_t)decpt);
    }
    return out;
}

struct Pose { double x, y, t; };

/* a grid of 9 m cells: every point within 8.5 m of (x, y) lies in the 3 x 3 cells around it */
struct Grid {
    static constexpr double kCell = 9.0;
    std::unordered_map<uint64_t, std::vector<uint32_t>> cells;
    static int64_t cell(double v) { return (int64_t)std::floor(v / kCell); }
    static uint64_t key(int64_t cx, int64_t cy) {
        return ((uint64_t)(uint32_t)(int32_t)cx << 32) | (uint64_t)(uint32_t)(int32_t)cy;
    }
    void add(double x, double y, uint32_t id) { cells[key(cell(x), cell(y))].push_back(id); }
    template <class F>
    void around(double x, double y, F &&f) const {
        const int64_t cx = cell(x), cy = cell(y);
        for (int64_t dx = -1; dx <= 1; dx++)
            for (int64_t dy = -1; dy <= 1; dy++) {
                auto it = cells.find(key(cx + dx, cy + dy));
                if (it == cells.end()) continue;
                for (uint32_t id : it->second)
                    if (!f(id)) return;
            }
    }
};

/* ---- generate_citytrees.py ---- */

/* its state_transition: heading unchanged when |omega| < 1e-10 */
Pose transition_citytrees(const Pose &p, double nu, double omega, double delta) {
    Pose n;
    if (std::fabs(omega) < 1e-10) {
        n.x = p.x + nu * std::cos(p.t) * delta;
        n.y = p.y + nu * std::sin(p.t) * delta;
        n.t = p.t;
    } else {
        n.x = p.x + nu / omega * (std::sin(p.t + omega * delta) - std::sin(p.t));
        n.y = p.y + nu / omega * (-std::cos(p.t + omega * delta) + std::cos(p.t));
        n.t = p.t + omega * delta;
    }
    return n;
}

struct Obs { int64_t step; int64_t lid; double r, b; };

int citytrees(int64_t n_poses, const char *path, uint64_t seed) {
    const double DELTA = 1.0, NU_MEAN = 1.0, NU_STD = 0.03, OMEGA_STD = 0.008;
    const int64_t BLOCK_MIN = 5, BLOCK_MAX = 75;
    const double SENSOR_RANGE = 8.5, LANDMARK_DENSITY = 3.0e-3, TURN_NU_SCALE = 1.12;
    const int64_t LANDMARK_STRIP_WIDTH = 20, MAX_OBS_PER_LM = 10;
    PyRandom rng(seed);

    /* phase 1: turn steps */
    std::map<int64_t, double> turns;
    for (int64_t step = 1; step < n_poses;) {
        step += rng.randint(BLOCK_MIN, BLOCK_MAX);
        if (step >= n_poses) break;
        const double turn_dir = rng.randbelow(2) == 0 ? -1.0 : 1.0;
        turns[step] = turn_dir * kPi / 2;
        step += 1;
    }

    /* phase 2: controls */
    std::vector<std::pair<double, double>> us;
    for (int64_t step = 1; step < n_poses; step++) {
        double nu, omega;
        auto it = turns.find(step);
        if (it != turns.end()) {
            omega = it->second / DELTA;
            nu = NU_MEAN * TURN_NU_SCALE + rng.gauss(0.0, NU_STD);
        } else {
            omega = rng.gauss(0.0, OMEGA_STD);
            nu = NU_MEAN + rng.gauss(0.0, NU_STD);
            const double lo = nu < 1.65 ? nu : 1.65;
            nu = lo > 0.85 ? lo : 0.85;
        }
        us.push_back({nu, omega});
    }

    /* phase 3: ground truth and dead reckoning */
    std::vector<Pose> gt{{0.0, 0.0, 0.0}}, poses{{0.0, 0.0, 0.0}};
    for (auto &u : us) {
        Pose n = transition_citytrees(gt.back(), u.first, u.second, DELTA);
        n.t = py_mod(n.t + kPi, 2 * kPi) - kPi;
        gt.push_back(n);
    }
    const double NN = 0.19, NO = 0.001, ON = 0.13, OO = 0.2;
    for (auto &u : us) {
        const double nu = u.first, omega = u.second;
        const double sigma_nu = std::sqrt(std::pow(NN, 2.0) * std::fabs(nu) + std::pow(NO, 2.0) * std::fabs(omega) + 1e-9);
        const double sigma_omega = std::sqrt(std::pow(ON, 2.0) * std::fabs(nu) + std::pow(OO, 2.0) * std::fabs(omega) + 1e-9);
        const double nu_noisy = nu + rng.gauss(0.0, sigma_nu);
        const double omega_noisy = omega + rng.gauss(0.0, sigma_omega);
        Pose n = transition_citytrees(poses.back(), nu_noisy, omega_noisy, DELTA);
        n.t = py_mod(n.t + kPi, 2 * kPi) - kPi;
        poses.push_back(n);
    }

    /* phase 4: landmarks in the bounding box, kept when a sampled pose sees them */
    double x_min = gt[0].x, x_max = gt[0].x, y_min = gt[0].y, y_max = gt[0].y;
    for (auto &p : gt) {
        if (p.x < x_min) x_min = p.x;
        if (p.x > x_max) x_max = p.x;
        if (p.y < y_min) y_min = p.y;
        if (p.y > y_max) y_max = p.y;
    }
    x_min -= (double)LANDMARK_STRIP_WIDTH; x_max += (double)LANDMARK_STRIP_WIDTH;
    y_min -= (double)LANDMARK_STRIP_WIDTH; y_max += (double)LANDMARK_STRIP_WIDTH;
    const double area = (x_max - x_min) * (y_max - y_min);
    const int64_t target = std::max<int64_t>(10, (int64_t)(area * LANDMARK_DENSITY));
    const int64_t stride = std::max<int64_t>(1, (int64_t)gt.size() / 500);
    Grid samples;
    for (int64_t i = 0; i < (int64_t)gt.size(); i += stride) samples.add(gt[i].x, gt[i].y, (uint32_t)i);
    const double range2 = std::pow(SENSOR_RANGE, 2.0);
    std::vector<std::pair<double, double>> lms;   /* id = 6 + index */
    for (int64_t attempts = 0; (int64_t)lms.size() < target && attempts < target * 50;) {
        attempts++;
        const double mx = rng.uniform(x_min, x_max);
        const double my = rng.uniform(y_min, y_max);
        bool visible = false;
        samples.around(mx, my, [&](uint32_t i) {
            if (std::pow(mx - gt[i].x, 2.0) + std::pow(my - gt[i].y, 2.0) <= range2) visible = true;
            return !visible;
        });
        if (visible) lms.push_back({mx, my});
    }

    /* phase 5: observations from the ground truth, each landmark at most 10 times */
    Grid lgrid;
    for (size_t k = 0; k < lms.size(); k++) lgrid.add(lms[k].first, lms[k].second, (uint32_t)k);
    std::vector<int64_t> count(lms.size(), 0);
    std::vector<Obs> obs;
    std::vector<uint32_t> cand;
    for (int64_t step = 0; step < (int64_t)gt.size(); step++) {
        const Pose &p = gt[step];
        cand.clear();
        lgrid.around(p.x, p.y, [&](uint32_t k) { cand.push_back(k); return true; });
        std::sort(cand.begin(), cand.end());
        for (uint32_t k : cand) {
            if (count[k] >= MAX_OBS_PER_LM) continue;
            const double dx = lms[k].first - p.x, dy = lms[k].second - p.y;
            const double dist = std::sqrt(dx * dx + dy * dy);
            if (dist > SENSOR_RANGE) continue;
            double bearing = std::atan2(dy, dx) - p.t;
            bearing = py_mod(bearing + kPi, 2 * kPi) - kPi;
            obs.push_back({step, 6 + (int64_t)k, dist, bearing});
            count[k]++;
        }
    }

    /* write_log */
    FILE *f = fopen(path, "w");
    if (!f) { fprintf(stderr, "gslam-data: cannot write %s\n", path); return 1; }
    fprintf(f, "delta %s\n", py_repr(DELTA).c_str());
    size_t q = 0;
    for (int64_t step = 0; step < n_poses; step++) {
        const double nu = step > 0 ? us[step - 1].first : 0.0, om = step > 0 ? us[step - 1].second : 0.0;
        fprintf(f, "u %lld %s %s\n", (long long)step, py_repr(nu).c_str(), py_repr(om).c_str());
        fprintf(f, "x %lld %s %s %s\n", (long long)step, py_repr(poses[step].x).c_str(),
                py_repr(poses[step].y).c_str(), py_repr(poses[step].t).c_str());
        for (; q < obs.size() && obs[q].step == step; q++)
            fprintf(f, "z %lld %lld %s %s\n", (long long)step, (long long)obs[q].lid, py_repr(obs[q].r).c_str(),
                    py_repr(obs[q].b).c_str());
    }
    fclose(f);
    std::vector<bool> seen(lms.size(), false);
    int64_t n_lm = 0;
    for (auto &o : obs)
        if (!seen[o.lid - 6]) { seen[o.lid - 6] = true; n_lm++; }
    printf("Generated %s\n", path);
    printf("  Poses: %lld, Landmarks: %lld, Observations: %lld, dim: %lld\n", (long long)n_poses,
           (long long)n_lm, (long long)obs.size(), (long long)(n_poses * 3));
    return 0;
}

/* ---- convert_slampp.py ---- */

/* its state_transition: heading advanced by omega * delta in both branches */
Pose transition_slampp(const Pose &p, double nu, double omega, double delta) {
    Pose n;
    if (std::fabs(omega) < 1e-10) {
        n.x = p.x + nu * std::cos(p.t) * delta;
        n.y = p.y + nu * std::sin(p.t) * delta;
    } else {
        n.x = p.x + nu / omega * (std::sin(p.t + omega * delta) - std::sin(p.t));
        n.y = p.y + nu / omega * (-std::cos(p.t + omega * delta) + std::cos(p.t));
    }
    n.t = p.t + omega * delta;
    return n;
}

bool parse_int(const std::string &s, int64_t *v) {
    char *end = nullptr;
    errno = 0;
    const long long x = strtoll(s.c_str(), &end, 10);
    if (errno || end == s.c_str() || *end) return false;
    *v = x;
    return true;
}

bool parse_float(const std::string &s, double *v) {
    char *end = nullptr;
    const double x = strtod(s.c_str(), &end);
    if (end == s.c_str() || *end) return false;
    *v = x;
    return true;
}

int slampp(const char *in_path, const char *out_path, double delta) {
    FILE *in = fopen(in_path, "r");
    if (!in) { fprintf(stderr, "gslam-data: cannot read %s\n", in_path); return 1; }
    std::map<int64_t, std::array<double, 3>> odometry;
    struct Lm { int64_t pose, id; double r, b; };
    std::vector<Lm> landmarks;
    std::string line;
    int ch;
    int64_t lineno = 0;
    bool more = true;
    while (more) {
        line.clear();
        while ((ch = fgetc(in)) != EOF && ch != '\n') line += (char)ch;
        more = (ch != EOF);
        if (!more && line.empty()) break;
        lineno++;
        std::vector<std::string> parts;
        size_t i = 0;
        while (i < line.size()) {
            while (i < line.size() && isspace((unsigned char)line[i])) i++;
            size_t j = i;
            while (j < line.size() && !isspace((unsigned char)line[j])) j++;
            if (j > i) parts.push_back(line.substr(i, j - i));
            i = j;
        }
        if (parts.empty()) continue;
        bool ok = true;
        if (parts[0] == "ODOMETRY") {
            int64_t from;
            std::array<double, 3> d{};
            ok = parts.size() >= 6 && parse_int(parts[1], &from) && parse_float(parts[3], &d[0]) &&
                 parse_float(parts[4], &d[1]) && parse_float(parts[5], &d[2]);
            if (ok) odometry[from] = d;
        } else if (parts[0] == "LANDMARK") {
            Lm l;
            ok = parts.size() >= 5 && parse_int(parts[1], &l.pose) && parse_int(parts[2], &l.id) &&
                 parse_float(parts[3], &l.r) && parse_float(parts[4], &l.b);
            if (ok) landmarks.push_back(l);
        }
        if (!ok) {
            fprintf(stderr, "gslam-data: %s:%lld: malformed %s record\n", in_path, (long long)lineno, parts[0].c_str());
            fclose(in);
            return 1;
        }
    }
    fclose(in);
    if (odometry.empty()) { fprintf(stderr, "gslam-data: %s has no ODOMETRY records\n", in_path); return 1; }
    const int64_t n_poses = odometry.rbegin()->first + 2;
    if (n_poses < 1) { fprintf(stderr, "gslam-data: negative pose ids in %s\n", in_path); return 1; }
    std::vector<Pose> poses((size_t)n_poses, Pose{0.0, 0.0, 0.0});
    std::vector<std::pair<double, double>> us((size_t)n_poses, {0.0, 0.0});
    for (int64_t step = 0; step < n_poses - 1; step++) {
        auto it = odometry.find(step);
        if (it == odometry.end()) {
            poses[step + 1] = poses[step];
            continue;
        }
        const double dx = it->second[0], dy = it->second[1], dtheta = it->second[2];
        const double nu = std::sqrt(dx * dx + dy * dy), omega = dtheta;
        poses[step + 1] = transition_slampp(poses[step], nu, omega, delta);
        us[step + 1] = {nu, omega};
    }
    FILE *out = fopen(out_path, "w");
    if (!out) { fprintf(stderr, "gslam-data: cannot write %s\n", out_path); return 1; }
    fprintf(out, "delta %s\n", py_repr(delta).c_str());
    for (int64_t step = 0; step < n_poses; step++) {
        fprintf(out, "u %lld %s %s\n", (long long)step, py_repr(us[step].first).c_str(), py_repr(us[step].second).c_str());
        fprintf(out, "x %lld %s %s %s\n", (long long)step, py_repr(poses[step].x).c_str(),
                py_repr(poses[step].y).c_str(), py_repr(poses[step].t).c_str());
    }
    for (auto &l : landmarks)
        fprintf(out, "z %lld %lld %s %s\n", (long long)l.pose, (long long)l.id, py_repr(l.r).c_str(),
                py_repr(l.b).c_str());
    fclose(out);
    printf("Converted %s -> %s\n", in_path, out_path);
    printf("  Poses: %lld, Observations: %lld, dim: %lld\n", (long long)n_poses, (long long)landmarks.size(),
           (long long)(n_poses * 3));
    return 0;
}

int usage(const char *argv0) {
    fprintf(stderr,
            "Usage: %s citytrees <n_poses> <output.txt> [seed=42]\n"
            "       %s slampp <input.txt> <output.log.txt> [delta=1.0]\n",
            argv0, argv0);
    return 1;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 4) return usage(argv[0]);
    if (strcmp(argv[1], "citytrees") == 0) {
        int64_t n = 0, seed = 42;
        if (!parse_int(argv[2], &n) || n < 1 || (argc > 4 && !parse_int(argv[4], &seed)))
            return usage(argv[0]);
        return citytrees(n, argv[3], (uint64_t)(seed < 0 ? -seed : seed));
    }
    if (strcmp(argv[1], "slampp") == 0) {
        double delta = 1.0;
        if (argc > 4 && !parse_float(argv[4], &delta)) return usage(argv[0]);
        return slampp(argv[2], argv[3], delta);
    }
    return usage(argv[0]);
}
