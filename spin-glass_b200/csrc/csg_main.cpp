// csg_main.cpp — the `csg <sim_dir> <H>` command on top of libcsg.so.
//
// Drop-in for the reference program's main (Program/src/main.cu:8-84): same
// arguments, same files in <sim_dir> (<H>-chkpt.bin read if present and
// rewritten at the end, <H>-obs.bin appended with obs_s records
// [sections][NDIS][NREP], eamsim.cuh:55-62), same log file <unix time>.log in
// the working directory, removed on success, same exit codes.
//
// Defaults are the reference's compile-time constants (eamsim.cuh:13-22):
// L=16, NDIS=2048, NCP=2, NREP=24, SBSHFL=16, SBMEAS=1024, SPFILE=262144,
// beta_r = 2 (2^(-4/23))^r.  An optional <sim_dir>/csg.conf (key = value
// lines: L, NDIS, NREP, SBSHFL, SBMEAS, SPFILE, seed, beta_max, beta_min)
// changes them.  Next to the checkpoint, <H>-chkpt.csg records the sweep
// counter and the seed, so that a resumed run continues the same Markov chain
// bit for bit; a reference checkpoint without it starts a new chain.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "csg.h"

namespace {

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Timestamped log to stdout and the log file (util.cu:22-47).
class Log {
  public:
    void open(const std::string& path) {
        path_ = path;
        f_.open(path, std::ios::app);
    }
    void record(const std::string& msg) {
        char ts[32];
        const time_t now = time(nullptr);
        strftime(ts, sizeof ts, "[%d/%m/%y %H:%M:%S] ", localtime(&now));
        if (f_.is_open()) f_ << ts << msg << std::endl;
        std::cout << ts << msg << std::endl;
    }
    void progress(double pc) {
        std::ostringstream s;
        s << "progress: " << std::setw(5) << std::setfill('0') << std::fixed << std::setprecision(1)
          << pc << "%";
        std::cout << s.str() << "\r" << std::flush;
    }
    void remove_file() {
        f_.close();
        std::remove(path_.c_str());
    }

  private:
    std::string path_;
    std::ofstream f_;
};

std::string fixed(double v, int width, int prec) {
    std::ostringstream s;
    s << std::setw(width) << std::setfill('0') << std::fixed << std::setprecision(prec) << v;
    return s.str();
}

void check(int rc, const char* what) {
    if (rc != CSG_OK) throw Error(std::string(what) + ": " + csg_last_error());
}

struct Settings {
    int L = 16, ndis = 2048, nrep = 24, sbshfl = 16, sbmeas = 1024;
    int64_t spfile = 262144;
    uint64_t seed = 0;
    bool seed_given = false;
    double beta_max = 2.0, beta_min = 0.125;
};

Settings read_settings(const std::string& sim_dir) {
    Settings st;
    std::ifstream f(sim_dir + "/csg.conf");
    if (!f.is_open()) return st;
    std::string line;
    while (std::getline(f, line)) {
        const auto hash = line.find('#');
        if (hash != std::string::npos) line.erase(hash);
        const auto eq = line.find('=');
        if (eq == std::string::npos) continue;
        std::string k = line.substr(0, eq), v = line.substr(eq + 1);
        auto trim = [](std::string& x) {
            x.erase(0, x.find_first_not_of(" \t"));
            x.erase(x.find_last_not_of(" \t\r") + 1);
        };
        trim(k);
        trim(v);
        if (k == "L") st.L = std::stoi(v);
        else if (k == "NDIS") st.ndis = std::stoi(v);
        else if (k == "NREP") st.nrep = std::stoi(v);
        else if (k == "SBSHFL") st.sbshfl = std::stoi(v);
        else if (k == "SBMEAS") st.sbmeas = std::stoi(v);
        else if (k == "SPFILE") st.spfile = std::stoll(v);
        else if (k == "seed") { st.seed = std::stoull(v, nullptr, 0); st.seed_given = true; }
        else if (k == "beta_max") st.beta_max = std::stod(v);
        else if (k == "beta_min") st.beta_min = std::stod(v);
        else throw Error("unknown key in csg.conf: " + k);
    }
    if (st.ndis % 32 || st.ndis <= 0) throw Error("NDIS must be a positive multiple of 32");
    if (st.sbmeas <= 0 || st.spfile % st.sbmeas) throw Error("SPFILE must be a multiple of SBMEAS");
    return st;
}

bool file_exists(const std::string& p) {
    std::ifstream f(p, std::ios::binary);
    return f.good();
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) { std::cout << "missing arguments\n"; return EXIT_FAILURE; }
    if (argc > 3) { std::cout << "extra arguments\n"; return EXIT_FAILURE; }
    const std::string sim_dir = argv[1];
    float H = 0.f;
    try {
        H = std::stof(argv[2]);
    } catch (const std::exception&) {
        std::cout << "invalid H\n";
        return EXIT_FAILURE;
    }
    const std::string base = sim_dir + "/" + fixed(H, 6, 4) + "-";
    const time_t t_s = time(nullptr);
    Log log;
    log.open(std::to_string(t_s) + ".log");
    csg_engine* e = nullptr;
    try {
        if (!(0.0f <= H && H <= 4.0f)) throw Error("H out of range");
        log.record("H = " + fixed(H, 6, 4));
        const Settings st = read_settings(sim_dir);
        std::vector<double> betas(st.nrep);
        for (int r = 0; r < st.nrep; ++r) {
            const double ratio = std::pow(st.beta_min / st.beta_max, 1.0 / (st.nrep - 1));
            betas[r] = (double)(float)(std::pow(ratio, r) * st.beta_max);
        }
        // resume state
        int64_t sweep = 0;
        uint64_t seed = st.seed_given ? st.seed : (uint64_t)t_s;
        const bool prev_sim = file_exists(base + "chkpt.bin");
        if (prev_sim && file_exists(base + "chkpt.csg")) {
            std::ifstream sc(base + "chkpt.csg");
            std::string magic;
            uint64_t s_seed = 0;
            int64_t s_sweep = 0;
            sc >> magic >> s_sweep >> s_seed;
            if (magic != "csg-resume-v1" || s_sweep < 0) throw Error("bad resume sidecar");
            sweep = s_sweep;
            seed = s_seed;
        }
        csg_config cfg{};
        cfg.dims = {st.L, st.ndis / 32, 2, st.nrep};
        cfg.sched = {st.sbshfl, st.sbmeas, 0};
        cfg.H = H;
        cfg.seed = seed;
        cfg.betas = betas.data();
        cfg.flags = CSG_MEASURE_M;
        check(csg_engine_create(&cfg, &e), "engine");
        log.record("eamsim initialized");

        const size_t N = (size_t)st.L * st.L * st.L;
        const size_t nref = (size_t)2 * st.ndis * N;
        std::vector<uint32_t> ref(nref);
        if (!prev_sim) {
            check(csg_init_lattice(e), "init");
            log.record("lattice array initialized");
        } else {
            std::ifstream f(base + "chkpt.bin", std::ios::binary);
            if (!f.is_open()) throw Error("unable to open " + base + "chkpt.bin");
            f.read(reinterpret_cast<char*>(ref.data()), (std::streamsize)(nref * 4));
            if ((size_t)f.gcount() != nref * 4) throw Error("checkpoint is truncated");
            check(csg_load_checkpoint(e, ref.data(), nref, sweep), "checkpoint");
            log.record("checkpoint loaded");
        }

        std::ofstream out(base + "obs.bin", std::ios::binary | std::ios::app);
        if (!out.is_open()) throw Error("unable to open " + base + "obs.bin");
        const size_t nrec = (size_t)st.ndis * st.nrep * 11;
        std::vector<float> rec(nrec);
        const auto t0 = std::chrono::steady_clock::now();
        // csg_run only queues the section on the GPU: the next section is
        // queued as soon as this one's records are taken, so that writing them
        // to the file overlaps the GPU's work
        check(csg_run(e, st.sbmeas), "run");
        for (int64_t done = 0; done < st.spfile; done += st.sbmeas) {
            log.progress(100.0 * (double)done / (double)st.spfile);
            check(csg_obs_records(e, rec.data(), nrec), "observables");
            if (done + st.sbmeas < st.spfile) check(csg_run(e, st.sbmeas), "run");
            out.write(reinterpret_cast<const char*>(rec.data()), (std::streamsize)(nrec * 4));
            if (!out) throw Error("write to " + base + "obs.bin failed");
        }
        out.close();
        const double secs =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        const double t_e = secs * 1e12 / ((double)st.spfile * N * 2 * st.ndis * st.nrep);
        // the reference prints %05.2f (util.cu); at this speed two decimals hold
        // about one significant digit, so four are printed
        log.record("t_e = " + fixed(t_e, 7, 4) + " ps");
        log.record("simulation ended");

        check(csg_save_checkpoint(e, ref.data(), nref), "checkpoint");
        std::ofstream f(base + "chkpt.bin", std::ios::binary);
        if (!f.is_open()) throw Error("unable to open " + base + "chkpt.bin");
        f.write(reinterpret_cast<const char*>(ref.data()), (std::streamsize)(nref * 4));
        if (!f) throw Error("write to " + base + "chkpt.bin failed");
        f.close();
        std::ofstream sc(base + "chkpt.csg");
        sc << "csg-resume-v1 " << sweep + st.spfile << " " << seed << "\n";
        if (!sc) throw Error("write to " + base + "chkpt.csg failed");
        log.record("checkpoint saved");
    } catch (const std::exception& err) {
        log.record(err.what());
        csg_engine_destroy(e);
        return EXIT_FAILURE;
    }
    csg_engine_destroy(e);
    log.remove_file();
    return EXIT_SUCCESS;
}
