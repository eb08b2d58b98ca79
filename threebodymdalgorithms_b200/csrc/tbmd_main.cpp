// tbmd_main: drop-in replacement for the reference's `main` executable, running the AT three-body
// Simulation on one GPU through the C ABI (include/tbmd.h).
//
// CLI (src/utility/cli.hpp:47-187): -a|--algorithm nata|auta|p3bca, -i|--iterations, -d|--delta,
// -c|--cutoff, -gx/-gy/-gz|--gravityX/Y/Z, -csv|--csv, -o|--out, -op|--outProfile,
// -decomp|--decomp optimal|naive, -benchyaml|--benchyaml.  Same parsing rules: a flag without a
// value or a value that does not convert prints the help and exits 1, an unknown option is
// reported and skipped, unset values are 0 and the algorithm defaults to NATA (the reference's
// zero-initialised globals, main.cpp:27).  Upper-case algorithm names are accepted as well.
// -benchyaml is accepted and ignored.  -np P lays the run out as the reference would on P MPI
// ranks (tbmd_rank_layout_of: process grid from -decomp, P3BCA's cutoff-window check, AtomDecomposition
// padding) and stops where that run stops, with its message and exit status 1; the GPU run itself is
// the same for every P.  -layoutonly prints that layout as JSON and exits without touching the GPU.
// GPU options: -prec fp64|mixed, -nu V (AT strength, default 1.0 as main.cpp:41), -device N,
// -nograph, -tune CACHE.JSONL (autotuner), -dumpfull FILE (state at %.17g after the run),
// -checkpoint FILE (the state after the run as an input CSV at 17 digits: -csv FILE resumes exactly),
// -parseonly (print the parsed arguments as JSON and exit without touching the GPU).
// -op FILE writes the profile document of the reference's PROFILE_3BMDA build (main.cpp:127-451):
// "times" per timer (time unit, avg/total over ranks, per-rank lists), "hitrate" (triplets inside
// over the C(N,3) candidates the reference's P=1 loop visits, per step), "hitrate per proc" and
// "stvr", with the GPU phases as timers (one rank).  -opsteps FILE writes per-step times in the
// MEASURESIMSTEP_3BMDA line format (Simulation.cpp:59-68, nanoseconds) plus the triplet count.
//
// Output (Simulation.cpp:74-79, utility.cpp:54-68): with -o base.csv, after every step i the file
// base_<i>.csv with header "ID, pX, pY, pZ, vX, vY, vZ, aX, aY, aZ, m, fX, fY, fZ", rows sorted by
// ID, values in the default ostream format (6 significant digits).
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <numeric>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "tbmd.h"

namespace {

struct Args {
    int iterations = 0;
    double cutoff = 0.0;
    double deltaT = 0.0;
    std::string inputCSV, outputCSV, outputProfile, outputSteps, benchYaml;
    int algorithm = TBMD_NATA;
    double g[3] = {0.0, 0.0, 0.0};
    bool optimalDecomposition = false;
    int ranks = 1;            // -np: MPI ranks of the reference run being reproduced
    bool layoutOnly = false;  // -layoutonly
    bool inputSummary = false;  // -inputsummary
    // GPU options
    int precision = TBMD_FP64;
    double nu = 1.0;
    int device = 0;
    bool graph = true;
    bool parseOnly = false;
    std::string tuneCache, dumpFull, checkpoint;
};

// The first 15 lines are the reference's help text byte for byte (cli.hpp:27-45), including its
// "-gx,--gravityZ" label (the parser itself accepts --gravityX, as the reference's does), so that
// scripts that read the reference's output read this one too.  This build's own options follow.
void printHelp()
{
    std::cout << "Help: \n"
              << "Options:\n"
              << "\t-h,--help\t\tShow this help message\n"
              << "\t-a,--algorithm\t\talgorithm to use (\"nata\", \"p3bca\", \"auta\")\n"
              << "\t-i,--iterations\t\tnum of iterations to simulate\n"
              << "\t-d,--delta\t\tduration of one simulation step\n"
              << "\t-gx,--gravityZ\t\tgravitational force in x-direction\n"
              << "\t-gy,--gravityY\t\tgravitational force in y-direction\n"
              << "\t-gz,--gravityZ\t\tgravitational force in z-direction\n"
              << "\t-csv,--csv\t\tcsv file with particles\n"
              << "\t-o,--out\t\tcsv base file name that will be used to create all csv outputs from each "
                 "simulation step\n"
              << "-op,--outProfile\t\tjson file to save profile output\n"
              << "-decomp,--decomp\t\t(optimal | naive) decomposition strategy for cart topology\n"
              << "-benchyaml,--benchyaml\t\tYAML file that contains config for benchmarks\n"
              << "\t-c,--cutoff\t\tcutoff distance\n"
              << "Notes: -decomp applies with -np; -benchyaml is accepted and ignored.\n"
              << "GPU options:\n"
              << "\t-prec\t\tfp64 | mixed\n\t-nu\t\tAT strength (1.0)\n\t-device\t\tCUDA device\n"
              << "\t-nograph\t\tno CUDA graph\n\t-tune\t\tautotuner cache file\n"
              << "\t-dumpfull\t\twrite the final state with 17 digits\n"
              << "\t-checkpoint\t\twrite the final state as an input CSV with 17 digits (restart with -csv)\n"
              << "\t-opsteps\t\tper-step timings (json lines)\n"
              << "\t-parseonly\t\tprint parsed args\n"
              << "\t-np\t\tMPI ranks of the reference run to reproduce (layout and checks; default 1)\n"
              << "\t-layoutonly\t\tprint the rank layout as JSON and exit\n"
              << "\t-inputsummary\t\tprint what was read from -csv as JSON and exit" << std::endl;
}

[[noreturn]] void usageExit()
{
    printHelp();
    std::exit(1);
}

bool isFlag(const std::string &f, const char *shortName, const char *longName)
{
    return f == shortName || f == longName;
}

Args parse(const std::vector<std::string> &args)
{
    Args a;
    for (size_t i = 0; i < args.size(); ++i) {
        try {
            if (args[i].rfind("-", 0) != 0) {
                std::cout << "CLI parser: unrecognized option: " << args[i] << std::endl;
                continue;
            }
            const std::string f = args[i].substr(1);
            auto value = [&]() -> std::string {
                if (args.size() <= i + 1) usageExit();
                return args[++i];
            };
            if (isFlag(f, "c", "-cutoff")) {
                a.cutoff = std::stod(value());
            } else if (isFlag(f, "i", "-iterations")) {
                a.iterations = std::stoi(value());
            } else if (isFlag(f, "a", "-algorithm")) {
                std::string v = value();
                if (v == "nata" || v == "NATA") a.algorithm = TBMD_NATA;
                else if (v == "p3bca" || v == "P3BCA") a.algorithm = TBMD_P3BCA;
                else if (v == "auta" || v == "AUTA") a.algorithm = TBMD_AUTA;
                else usageExit();
            } else if (isFlag(f, "decomp", "-decomp")) {
                std::string v = value();
                if (v == "optimal") a.optimalDecomposition = true;
                else if (v == "naive") a.optimalDecomposition = false;
                else usageExit();
            } else if (isFlag(f, "d", "-delta")) {
                a.deltaT = std::stod(value());
            } else if (isFlag(f, "csv", "-csv")) {
                a.inputCSV = value();
            } else if (isFlag(f, "o", "-out")) {
                a.outputCSV = value();
            } else if (isFlag(f, "op", "-outProfile")) {
                a.outputProfile = value();
            } else if (isFlag(f, "benchyaml", "-benchyaml")) {
                a.benchYaml = value();
            } else if (isFlag(f, "gx", "-gravityX")) {
                a.g[0] = std::stod(value());
            } else if (isFlag(f, "gy", "-gravityY")) {
                a.g[1] = std::stod(value());
            } else if (isFlag(f, "gz", "-gravityZ")) {
                a.g[2] = std::stod(value());
            } else if (isFlag(f, "prec", "-precision")) {
                std::string v = value();
                if (v == "fp64") a.precision = TBMD_FP64;
                else if (v == "mixed") a.precision = TBMD_MIXED;
                else usageExit();
            } else if (isFlag(f, "nu", "-nu")) {
                a.nu = std::stod(value());
            } else if (isFlag(f, "device", "-device")) {
                a.device = std::stoi(value());
            } else if (isFlag(f, "nograph", "-nograph")) {
                a.graph = false;
            } else if (isFlag(f, "tune", "-tune")) {
                a.tuneCache = value();
            } else if (isFlag(f, "dumpfull", "-dumpfull")) {
                a.dumpFull = value();
            } else if (isFlag(f, "checkpoint", "-checkpoint")) {
                a.checkpoint = value();
            } else if (isFlag(f, "opsteps", "-opsteps")) {
                a.outputSteps = value();
            } else if (isFlag(f, "parseonly", "-parseonly")) {
                a.parseOnly = true;
            } else if (isFlag(f, "np", "-np")) {
                a.ranks = std::stoi(value());
                if (a.ranks < 1) usageExit();
            } else if (isFlag(f, "layoutonly", "-layoutonly")) {
                a.layoutOnly = true;
            } else if (isFlag(f, "inputsummary", "-inputsummary")) {
                a.inputSummary = true;
            } else if (isFlag(f, "h", "-help")) {
                printHelp();
                std::exit(0);
            } else {
                std::cout << "CLI parser: unrecognized option: " << f << std::endl;
            }
        } catch (std::exception &) {
            usageExit();
        }
    }
    return a;
}

struct Particles {
    std::vector<int32_t> id;
    std::vector<double> col[10];  // x y z vx vy vz ax ay az m
};

// utility.cpp:14-24: header row, then ID and 10 numeric columns; further columns are ignored.  Blank
// lines are skipped (and not counted as rows), a trailing carriage return is dropped, each cell is
// read with strtol / strtod from its start (leading blanks allowed), and the first bad row is
// reported.  The file is read at once and its rows are parsed by several threads.
bool readCSV(const std::string &path, Particles &p, std::string &err)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    std::string buf;
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size > 0) {
        buf.resize((size_t)size);
        const size_t got = std::fread(&buf[0], 1, (size_t)size, f);
        buf.resize(got);
    }
    std::fclose(f);
    // the rows: every non-blank line after the header, as [begin, end) without the line break
    std::vector<std::pair<size_t, size_t>> rows;
    size_t pos = buf.find('\n');
    pos = pos == std::string::npos ? buf.size() : pos + 1;  // skip the header line
    while (pos < buf.size()) {
        size_t e = buf.find('\n', pos);
        if (e == std::string::npos) e = buf.size();
        size_t le = e;
        if (le > pos && buf[le - 1] == '\r') --le;
        if (buf.find_first_not_of(" \t", pos) < le) rows.emplace_back(pos, le);
        pos = e + 1;
    }
    const size_t n = rows.size();
    p.id.assign(n, 0);
    for (auto &c : p.col) c.assign(n, 0.0);
    struct Bad {
        size_t row = SIZE_MAX;
        std::string msg;
    };
    auto parse = [&](size_t r0, size_t r1, Bad &bad) {
        for (size_t r = r0; r < r1; ++r) {
            const char *b = buf.data() + rows[r].first, *e = buf.data() + rows[r].second;
            const char *cell[11];
            int nc = 0;
            for (const char *q = b; nc < 11;) {
                cell[nc++] = q;
                q = (const char *)std::memchr(q, ',', (size_t)(e - q));
                if (!q) break;
                ++q;
            }
            if (nc < 11) {
                bad = {r, "row " + std::to_string(r) + " has fewer than 11 columns"};
                return;
            }
            char *end = nullptr;
            const long idv = std::strtol(cell[0], &end, 10);
            if (end == cell[0]) {
                bad = {r, "row " + std::to_string(r) + ": bad ID"};
                return;
            }
            p.id[r] = (int32_t)idv;
            for (int k = 0; k < 10; ++k) {
                const double v = std::strtod(cell[k + 1], &end);
                if (end == cell[k + 1]) {
                    const char *ce = (const char *)std::memchr(cell[k + 1], ',', (size_t)(e - cell[k + 1]));
                    bad = {r, "row " + std::to_string(r) + ": bad number '" +
                                  std::string(cell[k + 1], ce ? ce : e) + "'"};
                    return;
                }
                p.col[k][r] = v;
            }
        }
    };
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t nt = std::max<size_t>(1, std::min<size_t>({hw ? hw : 1u, 16u, (n + 8191) / 8192}));
    std::vector<Bad> bads(nt);
    std::vector<std::thread> pool;
    for (size_t t = 1; t < nt; ++t) pool.emplace_back(parse, n * t / nt, n * (t + 1) / nt, std::ref(bads[t]));
    parse(0, n / nt, bads[0]);
    for (auto &th : pool) th.join();
    for (const Bad &bd : bads)
        if (bd.row != SIZE_MAX) {  // chunks are in row order: the first one found is the first bad row
            err = bd.msg;
            return false;
        }
    return true;
}

std::string stepPath(const std::string &base, int step)
{
    return base.substr(0, base.find_last_of('.')) + "_" + std::to_string(step) + ".csv";
}

struct State {
    std::vector<int32_t> id;
    std::vector<double> v[13];  // x y z vx vy vz ax ay az m fx fy fz
};

bool fetch(tbmd_ctx *ctx, int64_t n, State &s)
{
    s.id.resize(n);
    for (auto &c : s.v) c.resize(n);
    return tbmd_get_particles(ctx, s.id.data(), s.v[0].data(), s.v[1].data(), s.v[2].data(), s.v[3].data(),
                              s.v[4].data(), s.v[5].data(), s.v[6].data(), s.v[7].data(), s.v[8].data(),
                              s.v[9].data(), s.v[10].data(), s.v[11].data(), s.v[12].data()) == TBMD_OK;
}

// Rows in ID order (Simulation.cpp:127-128).  IDs do not change between steps, so the order is
// computed once.
std::vector<size_t> idOrder(const std::vector<int32_t> &id)
{
    std::vector<size_t> order(id.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return id[a] < id[b]; });
    return order;
}

// utility.cpp:54-68 (writeStepToCSVWithForces): the reference's header and columns, each value as
// std::ostream prints it by default.  The rows are formatted by several threads, each into its own
// stream with the same default formatting, and written in order.
void writeStepCSV(const std::string &path, const State &s, const std::vector<size_t> &order)
{
    const size_t n = order.size();
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t nt = std::max<size_t>(1, std::min<size_t>({hw ? hw : 1u, 16u, (n + 4095) / 4096}));
    std::vector<std::string> parts(nt);
    auto format = [&](size_t t) {
        std::ostringstream o;
        for (size_t r = n * t / nt; r < n * (t + 1) / nt; ++r) {
            const size_t i = order[r];
            o << s.id[i];
            for (int k = 0; k < 13; ++k) o << ", " << s.v[k][i];
            o << "\n";
        }
        parts[t] = o.str();
    };
    std::vector<std::thread> pool;
    for (size_t t = 1; t < nt; ++t) pool.emplace_back(format, t);
    format(0);
    for (auto &th : pool) th.join();
    std::ofstream out(path);
    out << "ID, pX, pY, pZ, vX, vY, vZ, aX, aY, aZ, m, fX, fY, fZ\n";
    for (const std::string &part : parts) out << part;
}

// The state as an input file of the reference's format (utility.cpp:14-24: header, then ID and the
// ten columns pX..pZ, vX..vZ, aX..aZ, m that the reader takes), with the forces appended as three more
// columns, which the reader ignores.  Every value at 17 significant digits, so reading it back with
// -csv restores the state exactly: an exact checkpoint, where the per-step output keeps the reference's
// 6 digits.  A restarted P3BCA run takes its periodic domain from these positions, as the reference's
// Init does for any input file (RegularGridDecomposition.cpp:135-166).
bool writeCheckpoint(const std::string &path, const State &s)
{
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    std::fprintf(f, "ID, pX, pY, pZ, vX, vY, vZ, aX, aY, aZ, m, fX, fY, fZ\n");
    for (size_t i = 0; i < s.id.size(); ++i) {
        std::fprintf(f, "%d", s.id[i]);
        for (int k = 0; k < 13; ++k) std::fprintf(f, ", %.17g", s.v[k][i]);
        std::fprintf(f, "\n");
    }
    return std::fclose(f) == 0;
}

void writeFull(const std::string &path, const State &s, const std::vector<uint64_t> &counts)
{
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) return;
    for (size_t i = 0; i < counts.size(); ++i)
        std::fprintf(f, "step %zu buffer 1 triplets %llu\n", i, (unsigned long long)counts[i]);
    for (size_t i = 0; i < s.id.size(); ++i) {
        std::fprintf(f, "particle %d", s.id[i]);
        for (int k = 0; k < 13; ++k) std::fprintf(f, " %.17g", s.v[k][i]);
        std::fprintf(f, "\n");
    }
    std::fclose(f);
}

}  // namespace

// The PROFILE_3BMDA document (main.cpp:127-451) for one rank.  Timers are the GPU phases of a step
// (device time per step, nanoseconds); the reference's force timer name "calculateForces" is the
// triplet phase, and "simulationStep" is the host wall time of the whole step.  hitrate: triplets
// inside over C(N,3), the candidates of the reference's P=1 loop (P3BCA.cpp:632-636, 790-794).
// stvr of a single rank is 0.
static void writeProfile(const std::string &path, const std::vector<std::vector<long long>> &phaseNs,
                         const std::vector<long long> &stepNs, const std::vector<uint64_t> &counts, int64_t n)
{
    static const char *names[] = {"predictor", "cellBuild", "neighbourLists", "calculateForces", "update"};
    std::ofstream o(path);
    o << "{\"times\": {";
    const size_t nphase = phaseNs.empty() ? 0 : std::min<size_t>(phaseNs[0].size(), 5);
    for (size_t k = 0; k <= nphase; ++k) {
        std::vector<long long> v;
        for (size_t i = 0; i < stepNs.size(); ++i) v.push_back(k < nphase ? phaseNs[i][k] : stepNs[i]);
        long long total = 0;
        for (long long t : v) total += t;
        const double avg = v.empty() ? 0.0 : (double)total / (double)v.size();
        o << (k ? ", " : "") << "\"" << (k < nphase ? names[k] : "simulationStep")
          << "\": {\"time unit\": \"nanosecond\", \"avg time all proc\": " << avg
          << ", \"total time all proc\": " << (double)total << ", \"total avg time union proc\": " << (double)total
          << ", \"total max time union proc\": " << total << ", \"times per proc\": {\"0\": [";
        for (size_t i = 0; i < v.size(); ++i) o << (i ? ", " : "") << v[i];
        o << "]}}";
    }
    const double cand = n >= 3 ? (double)n * (double)(n - 1) * (double)(n - 2) / 6.0 : 0.0;
    std::ostringstream hr;
    hr.precision(17);
    for (size_t i = 0; i < counts.size(); ++i) hr << (i ? ", " : "") << (cand > 0 ? (double)counts[i] / cand : 0.0);
    o << "}, \"hitrate\": {\"avg hitrate per sim step\": [" << hr.str() << "]}, \"hitrate per proc\": {\"0\": ["
      << hr.str() << "]}, \"stvr\": [{\"rank\": [0], \"stvr\": 0.0}]}\n";
}

int main(int argc, char **argv)
{
    std::vector<std::string> args(argv + 1, argv + argc);
    Args a = parse(args);
    static const char *algName[3] = {"nata", "p3bca", "auta"};
    if (a.parseOnly) {
        std::printf("{\"algorithm\": \"%s\", \"iterations\": %d, \"delta\": %.17g, \"cutoff\": %.17g, "
                    "\"g\": [%.17g, %.17g, %.17g], \"csv\": \"%s\", \"out\": \"%s\", \"precision\": \"%s\", "
                    "\"nu\": %.17g, \"device\": %d, \"graph\": %s, \"ranks\": %d, \"decomp\": \"%s\"}\n",
                    algName[a.algorithm], a.iterations, a.deltaT, a.cutoff, a.g[0], a.g[1], a.g[2],
                    a.inputCSV.c_str(), a.outputCSV.c_str(), a.precision == TBMD_MIXED ? "mixed" : "fp64", a.nu,
                    a.device, a.graph ? "true" : "false", a.ranks, a.optimalDecomposition ? "optimal" : "naive");
        return 0;
    }
    if (!a.benchYaml.empty()) std::cout << "note: -benchyaml is ignored (no MPI benchmark harness)" << std::endl;

    Particles p;
    std::string err;
    if (!readCSV(a.inputCSV, p, err)) {
        std::cerr << "error reading particles: " << err << std::endl;
        return 1;
    }
    const int64_t n = (int64_t)p.id.size();
    if (a.inputSummary) {
        // what was read, for checks without a GPU: the row count, and per column the first, last,
        // smallest and largest value (%.17g), plus the ID sum
        long long idsum = 0;
        for (int32_t v : p.id) idsum += v;
        std::printf("{\"n\": %lld, \"id_sum\": %lld, \"columns\": [", (long long)n, idsum);
        for (int k = 0; k < 10; ++k) {
            const auto &c = p.col[k];
            const auto mm = n ? std::minmax_element(c.begin(), c.end()) : std::make_pair(c.begin(), c.begin());
            std::printf("%s[%.17g, %.17g, %.17g, %.17g]", k ? ", " : "", n ? c.front() : 0.0, n ? c.back() : 0.0,
                        n ? *mm.first : 0.0, n ? *mm.second : 0.0);
        }
        std::printf("]}\n");
        return 0;
    }

    if (a.ranks != 1 || a.layoutOnly) {
        // physical domain size as RegularGridDecomposition::getDomainMinMax takes it
        // (RegularGridDecomposition.cpp:135-166): the extent widened by 1e-4 on each side
        double L[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < 3 && n > 0; ++d) {
            const auto mm = std::minmax_element(p.col[d].begin(), p.col[d].end());
            L[d] = std::fabs((*mm.second + 0.0001) - (*mm.first - 0.0001));
        }
        tbmd_rank_layout lay;
        char msg[256];
        const tbmd_status ls = tbmd_rank_layout_of(a.algorithm, a.ranks, a.optimalDecomposition ? 1 : 0, a.cutoff,
                                                   L, n, &lay, msg, (int32_t)sizeof msg);
        if (ls == TBMD_RANK_LAYOUT) {
            std::cerr << msg << std::endl;
            return 1;
        }
        if (ls != TBMD_OK) {
            std::cerr << "error: " << tbmd_status_string(ls) << std::endl;
            return 1;
        }
        if (a.layoutOnly) {
            std::printf("{\"algorithm\": \"%s\", \"ranks\": %d, \"num_dims\": %d, \"dims\": [%d, %d, %d], "
                        "\"cutoff_boxes\": [%d, %d, %d], \"shift_steps\": %d, "
                        "\"cell_size\": [%.17g, %.17g, %.17g], \"particles_per_rank\": %lld, \"dummies\": %lld}\n",
                        algName[a.algorithm], lay.world_size, lay.num_dims, lay.dims[0], lay.dims[1], lay.dims[2],
                        lay.cutoff_boxes[0], lay.cutoff_boxes[1], lay.cutoff_boxes[2], lay.shift_steps,
                        lay.cell_size[0], lay.cell_size[1], lay.cell_size[2], (long long)lay.particles_per_rank,
                        (long long)lay.dummies);
            return 0;
        }
    }

    tbmd_config cfg;
    tbmd_config_init(&cfg);
    cfg.algorithm = a.algorithm;
    cfg.precision = a.precision;
    cfg.cutoff = a.algorithm == TBMD_P3BCA ? a.cutoff : 0.0;
    cfg.dt = a.deltaT;
    for (int d = 0; d < 3; ++d) cfg.g[d] = a.g[d];
    cfg.nu = a.nu;
    cfg.device = a.device;
    cfg.use_graph = a.graph ? 1 : 0;
    tbmd_ctx *ctx = nullptr;
    tbmd_status st = tbmd_create(&cfg, &ctx);
    if (st != TBMD_OK) {
        std::cerr << "error: " << tbmd_status_string(st) << std::endl;
        return 1;
    }
    auto die = [&](const char *what) {
        std::cerr << "error in " << what << ": " << tbmd_last_error(ctx) << std::endl;
        tbmd_destroy(ctx);
        std::exit(1);
    };
    if (n > 0) {
        const double *c = nullptr;
        (void)c;
        if (tbmd_set_particles(ctx, n, p.id.data(), p.col[0].data(), p.col[1].data(), p.col[2].data(),
                               p.col[3].data(), p.col[4].data(), p.col[5].data(), p.col[6].data(), p.col[7].data(),
                               p.col[8].data(), p.col[9].data()) != TBMD_OK)
            die("set_particles");
    }
    if (!a.tuneCache.empty() && n > 0 && tbmd_autotune(ctx, a.tuneCache.c_str()) != TBMD_OK) die("autotune");

    std::vector<uint64_t> counts;
    std::vector<long long> stepNs;
    std::vector<std::vector<long long>> phaseNs;  // [step][phase], device time of each GPU phase
    State s;
    State states[2];          // per-step CSV output: two host buffers, one being written out
    std::thread writer[2];
    std::vector<size_t> order;
    const bool profile = !a.outputProfile.empty();
    if (n > 0 && a.iterations > 0) {
        const bool perStep = !a.outputCSV.empty() || profile || !a.outputSteps.empty();
        if (perStep) {
            for (int i = 0; i < a.iterations; ++i) {
                uint64_t c = 0;
                if (profile && tbmd_set_profiling(ctx, 1) != TBMD_OK) die("set_profiling");  // resets the timers
                auto t0 = std::chrono::steady_clock::now();
                if (tbmd_step(ctx, 1, &c) != TBMD_OK) die("step");
                auto t1 = std::chrono::steady_clock::now();
                stepNs.push_back(std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
                counts.push_back(c);
                if (profile) {
                    double ms[8];
                    uint64_t calls[8], launches[8];
                    const int np = tbmd_phase_times(ctx, ms, calls, launches, 8);
                    std::vector<long long> row;
                    for (int k = 0; k < np; ++k) row.push_back((long long)(ms[k] * 1e6 + 0.5));
                    phaseNs.push_back(row);
                }
                if (!a.outputCSV.empty()) {
                    // the previous step's file is written in the background while this step ran;
                    // its buffer is fetched into again only after that write has finished
                    State &buf = states[i % 2];
                    if (writer[i % 2].joinable()) writer[i % 2].join();
                    if (!fetch(ctx, n, buf)) die("get_particles");
                    if (order.empty()) order = idOrder(buf.id);
                    writer[i % 2] = std::thread(writeStepCSV, stepPath(a.outputCSV, i), std::cref(buf), std::cref(order));
                }
            }
            for (auto &w : writer)
                if (w.joinable()) w.join();
            if (profile) tbmd_set_profiling(ctx, 0);
        } else {
            counts.resize(a.iterations);
            if (tbmd_step(ctx, a.iterations, counts.data()) != TBMD_OK) die("step");
        }
    }
    if (profile) writeProfile(a.outputProfile, phaseNs, stepNs, counts, n);
    if (!a.outputSteps.empty()) {
        std::ofstream prof(a.outputSteps);
        for (size_t i = 0; i < stepNs.size(); ++i)
            prof << "{\"allTimes\": [" << stepNs[i] << "], \"max\": " << stepNs[i] << ", \"triplets\": " << counts[i]
                 << "}\n";
    }
    if ((!a.dumpFull.empty() || !a.checkpoint.empty()) && n > 0) {
        if (!fetch(ctx, n, s)) die("get_particles");
        if (!a.dumpFull.empty()) writeFull(a.dumpFull, s, counts);
        if (!a.checkpoint.empty() && !writeCheckpoint(a.checkpoint, s)) die("checkpoint");
    }
    tbmd_destroy(ctx);
    return 0;
}
