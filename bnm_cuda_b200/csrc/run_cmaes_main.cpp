// run_CMAES_gpu: drop-in replacement for the reference driver (run_CMAES.cpp
// main(), GPU build) on top of the C ABI of libbnm_b200.
//
// Same command line (19 positional arguments, run_CMAES.cpp:192-218), BNM_*
// environment (constants.h:93-116), parameter expansion with optional
// regional maps (run_CMAES.cpp:61-143, 226-309), empirical FC/FCD input,
// output directories <out>/sims[_multimaps]_gpu and <out>/cmaes[_multimaps]_gpu,
// the CMA-ES log file and its lines (run_CMAES.cpp:417-445, 798-815, 821-906)
// and the best-simulation files (bnm.cu:771-833).
//
// Differences: analytic FIC runs on the device inside the batch call instead
// of per particle on the host; errors return a status instead of exit(1) deep
// inside the library.  BNM_B200_NOISE=philox switches the noise source from
// the reference's host stream (mt19937 + normal_distribution<float>) to the
// device Philox table; BNM_B200_PRECISION=f64|f32ref|f32 (default f32)
// selects the integrator arithmetic and BNM_B200_GRAM=f32|bf16|bf16x3 the FC /
// FCD Gram arithmetic (default bf16x3 with f32, f32 with the reference-order
// modes).
//
// Checkpoint / resume (no counterpart in the reference): with
// BNM_B200_CHECKPOINT=<file> the driver saves the CMA-ES state and the length
// of its log after every generation; a later run with the same arguments and
// file continues from there (the log is cut back to that length and
// appended), and gives the log and result files of an uninterrupted run.
// BNM_B200_MAX_GENERATIONS=<k> stops after k generations of this process
// (exit status 75, the checkpoint saved), for time-limited jobs.
// BNM_B200_METRICS=<file> appends one JSON line per generation (wall time,
// simulations per second, the device's stage times, the generation's best
// cost and the best fit so far).
#include <sys/stat.h>
#include <sys/types.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/bnm_b200.h"

namespace {

[[noreturn]] void die(const char* what) {
    std::fprintf(stderr, "Error: %s: %s\n", what, bnm_last_error());
    std::exit(1);
}

// helpers.cpp:4-11: doubles through float.
double env_f(const char* k, double d) {
    const char* v = std::getenv(k);
    return v ? (double)(float)std::atof(v) : d;
}

std::vector<double> read_numbers(const std::string& path, bool* ok) {
    std::ifstream f(path);
    std::vector<double> v;
    *ok = (bool)f;
    double x;
    while (f >> x) v.push_back(x);
    return v;
}

struct Driver {
    int nodes = 0, time_steps = 0, BOLD_TR = 0, window_size = 0, window_step = 0, rand_seed = 0;
    int lambda = 0, itMax = 0, SeedMW = 0;
    std::string sc_path, out_path, fc_tril_path, fcd_tril_path, maps_path, het_params_str;
    std::map<std::string, std::string> param_strings;
    std::map<std::string, double> params, param_mins, param_maxs, param_diffs;
    std::vector<std::string> free_params, het_params, homo_params;
    std::vector<std::vector<double>> maps;
    bool heterogeneous = false, do_fic = false;

    // run_CMAES.cpp:61-143, through the library's bnm_calculate_params
    void calculate_params(std::map<std::string, double>& cp, int ind, double* G, double* wEE, double* wEI,
                          double* wIE) const {
        static const char* kLocal[3] = {"wee", "wie", "wei"};  // run_CMAES.cpp:252
        int mask = 0;
        std::vector<double> scales(3 * std::max<size_t>(maps.size(), 1), 0.0), flat;
        for (int k = 0; k < 3; k++)
            if (std::find(het_params.begin(), het_params.end(), kLocal[k]) != het_params.end()) {
                mask |= 1 << k;
                for (size_t m = 0; m < maps.size(); m++)
                    scales[k * maps.size() + m] = cp[std::string(kLocal[k]) + "scale_" + std::to_string(m)];
            }
        for (auto& mp : maps) flat.insert(flat.end(), mp.begin(), mp.end());
        const size_t o = (size_t)ind * nodes;
        if (bnm_calculate_params(nodes, mask, (int)maps.size(), flat.empty() ? nullptr : flat.data(), cp["G"],
                                 cp["wee"], cp["wie"], cp["wei"], scales.data(), G + ind, wEE + o, wEI + o,
                                 wIE + o) != BNM_OK)
            die("calculate_params");
    }
};

void write_row(const std::string& path, const double* v, int n) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return;
    for (int j = 0; j < n; j++) std::fprintf(f, "%f ", v[j]);
    std::fclose(f);
}

// Driver checkpoint: one line "bnm_b200 driver checkpoint 1 <log bytes>"
// followed by the CMA-ES state as bnm_cmaes_save writes it; the file is
// written under a temporary name and renamed into place.
constexpr const char* kCkptTag = "bnm_b200 driver checkpoint 1";

bool slurp(const std::string& path, std::string* out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    *out = ss.str();
    return true;
}

bool write_checkpoint(const std::string& path, const bnm_cmaes* es, long log_bytes) {
    const std::string state = path + ".cmaes", tmp = path + ".tmp";
    std::string bytes;
    if (bnm_cmaes_save(es, state.c_str()) != 0 || !slurp(state, &bytes)) return false;
    std::remove(state.c_str());
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return false;
    bool ok = std::fprintf(f, "%s %ld\n", kCkptTag, log_bytes) > 0 &&
              std::fwrite(bytes.data(), 1, bytes.size(), f) == bytes.size() && std::fflush(f) == 0;
    ok = std::fclose(f) == 0 && ok;
    return ok && std::rename(tmp.c_str(), path.c_str()) == 0;
}

// 0: no checkpoint (a fresh run) or a checkpoint read into *es and *log_bytes;
// 1: a file that is not a driver checkpoint (reported).
int read_checkpoint(const std::string& path, bnm_cmaes** es, long* log_bytes) {
    std::string all;
    if (!slurp(path, &all)) return 0;
    const size_t nl = all.find('\n');
    const std::string tag = kCkptTag;
    char* end = nullptr;
    const long n = nl == std::string::npos || all.compare(0, tag.size(), tag) != 0
                       ? -1
                       : std::strtol(all.c_str() + tag.size(), &end, 10);
    const std::string state = path + ".cmaes";
    if (n >= 0 && end == all.c_str() + nl) {
        std::ofstream(state, std::ios::binary).write(all.data() + nl + 1, (std::streamsize)(all.size() - nl - 1));
        const int rc = bnm_cmaes_load(state.c_str(), es);
        std::remove(state.c_str());
        if (rc == 0) {
            *log_bytes = n;
            return 0;
        }
    }
    std::fprintf(stderr, "Error: %s is not a checkpoint of this driver\n", path.c_str());
    return 1;
}

}  // namespace

int main(int argc, char* argv[]) {
    Driver d;
    if (argc != 20) {
        std::printf(
            "Usage: ./run_CMAES_<cpu|gpu> <sc_path> <out_prefix|'same'> <fc_tril_path> <fcd_tril_path> <maps_path> "
            "<n_regions> <G_min[-G_max]> <wee_min[-wee_max]> <wei_min[-wei_max]> <wie_min[-wie_max]> <het_params> "
            "<time_steps> <BOLD_TR> <fcd_step> <fcd_window> <rand_seed> <lambda> <itMax> <SeedMW>\n");
        return 0;
    }
    d.sc_path = argv[1];
    d.out_path = argv[2];
    d.fc_tril_path = argv[3];
    d.fcd_tril_path = argv[4];
    d.maps_path = argv[5];
    d.nodes = std::atoi(argv[6]);
    d.param_strings["G"] = argv[7];
    d.param_strings["wee"] = argv[8];
    d.param_strings["wei"] = argv[9];
    d.param_strings["wie"] = argv[10];
    d.het_params_str = argv[11];
    d.time_steps = std::atoi(argv[12]);
    d.BOLD_TR = std::atoi(argv[13]);
    d.window_step = std::atoi(argv[14]);
    d.window_size = std::atoi(argv[15]);
    d.rand_seed = std::atoi(argv[16]);
    d.lambda = std::atoi(argv[17]);
    d.itMax = std::atoi(argv[18]);
    d.SeedMW = std::atoi(argv[19]);

    bnm_cmaes_params cp;
    bnm_cmaes_params_default(&cp);
    bnm_cmaes_params_from_env(&cp);
    int Dimension = 0;
    // free parameters: "min-max" (a leading '-' is a sign), run_CMAES.cpp:230-250
    for (auto& kv : d.param_strings) {
        std::string sub = kv.second.substr(1);
        size_t pos = sub.find('-');
        if (pos != std::string::npos) {
            d.params[kv.first] = -100;
            d.param_mins[kv.first] = std::atof(kv.second.substr(0, pos + 1).c_str());
            d.param_maxs[kv.first] = std::atof(kv.second.substr(pos + 2).c_str());
            d.param_diffs[kv.first] = d.param_maxs[kv.first] - d.param_mins[kv.first];
            Dimension++;
            d.free_params.push_back(kv.first);
        } else {
            d.params[kv.first] = std::atof(kv.second.c_str());
        }
    }
    for (std::string lp : {"wee", "wie", "wei"}) {
        if (d.het_params_str.find(lp) != std::string::npos) {
            d.heterogeneous = true;
            d.het_params.push_back(lp);
        } else {
            d.homo_params.push_back(lp);
        }
    }
    const double scale_max_minmax = env_f("BNM_SCALE_MAX_MINMAX", 1.0);
    if (d.heterogeneous) {  // run_CMAES.cpp:265-309
        std::ifstream mf(d.maps_path);
        if (!mf) {
            std::fprintf(stderr, "Error opening maps file\n");
            return 1;
        }
        std::string line;
        int idx = 0;
        while (std::getline(mf, line)) {
            std::vector<double> m;
            std::istringstream iss(line);
            double x;
            while (iss >> x) m.push_back(x);
            if (m.empty()) continue;
            double mx = *std::max_element(m.begin(), m.end()), mn = *std::min_element(m.begin(), m.end());
            double smin, smax;
            if (mn == 0 && mx == 1) {
                smin = 0;
                smax = scale_max_minmax;
            } else {
                smin = std::ceil((-1 / mx) / 0.01) * 0.01;
                smax = std::floor((-1 / mn) / 0.01) * 0.01;
            }
            d.maps.push_back(m);
            for (auto& h : d.het_params) {
                std::string name = h + "scale_" + std::to_string(idx);
                d.params[name] = -100;
                d.param_mins[name] = smin;
                d.param_maxs[name] = smax;
                d.param_diffs[name] = smax - smin;
                Dimension++;
                d.free_params.push_back(name);
            }
            idx++;
        }
    }
    bool ok;
    std::vector<double> emp_fc = read_numbers(d.fc_tril_path, &ok);
    if (!ok) {
        std::fprintf(stderr, "Error opening empirical FC file\n");
        return 1;
    }
    std::vector<double> emp_fcd;
    bool no_fcd = true;
    if (d.fcd_tril_path != "no_fcd") {
        emp_fcd = read_numbers(d.fcd_tril_path, &ok);
        if (!ok) {
            std::fprintf(stderr, "Error opening empirical FCD file\n");
            return 1;
        }
        no_fcd = false;
    }
    d.do_fic = (d.params["wie"] == 0);
    if (d.do_fic && std::find(d.het_params.begin(), d.het_params.end(), "wie") != d.het_params.end()) {
        std::fprintf(stderr, "Error: wIE cannot be a heterogeneous parameter in FIC+ model\n");
        return 1;
    }
    std::vector<double> sc((size_t)d.nodes * d.nodes);
    {
        FILE* fp = std::fopen(d.sc_path.c_str(), "r");
        if (!fp) {
            std::printf("Error opening SC file\n");
            return 1;
        }
        for (auto& v : sc)
            if (std::fscanf(fp, "%lf", &v) != 1) {
                std::printf("Error reading SC file\n");
                return 1;
            }
        std::fclose(fp);
    }

    // output locations, run_CMAES.cpp:398-430
    if (d.out_path == "same") d.out_path = d.sc_path.substr(0, d.sc_path.length() - 4);
    mkdir(d.out_path.c_str(), 0751);
    std::string sims_dir = d.out_path + "/sims", cmaes_dir = d.out_path + "/cmaes";
    if (d.heterogeneous) {
        sims_dir += "_multimaps";
        cmaes_dir += "_multimaps";
    }
    sims_dir += "_gpu";
    cmaes_dir += "_gpu";
    mkdir(sims_dir.c_str(), 0751);
    mkdir(cmaes_dir.c_str(), 0751);
    size_t pos = d.fc_tril_path.find_last_of('/');
    std::string prefix = d.fc_tril_path.substr(pos + 1, d.fc_tril_path.length() - pos - 17);
    for (auto& kv : d.param_strings) prefix += "_" + kv.first + "_" + kv.second;
    prefix += "_het-" + d.het_params_str + "_SeedMW-" + std::to_string(d.SeedMW) + "_SeedSim-" +
              std::to_string(d.rand_seed) + "_n-" + std::to_string(d.itMax) + "x" + std::to_string(d.lambda);
    const std::string log_path = cmaes_dir + "/" + prefix + ".txt", sims_prefix = sims_dir + "/" + prefix + "_";
    const char* ckpt_env = std::getenv("BNM_B200_CHECKPOINT");
    const std::string ckpt = ckpt_env ? ckpt_env : "";
    long resume_log_bytes = -1;
    bnm_cmaes* resumed = nullptr;
    if (!ckpt.empty() && read_checkpoint(ckpt, &resumed, &resume_log_bytes)) return 1;
    if (resumed && truncate(log_path.c_str(), (off_t)resume_log_bytes) != 0) {
        std::fprintf(stderr, "Error: cannot cut the log %s back to its checkpointed length\n", log_path.c_str());
        return 1;
    }
    FILE* log = std::fopen(log_path.c_str(), resumed ? "a" : "w");
    if (!log) {
        std::fprintf(stderr, "Error opening log file %s\n", log_path.c_str());
        return 1;
    }
    auto both = [&](const char* fmt, auto... a) {
        std::fprintf(log, fmt, a...);
        std::printf(fmt, a...);
    };
    auto header = [&](const char* fmt, auto... a) {  // already in a resumed log
        if (!resumed) std::fprintf(log, fmt, a...);
        std::printf(fmt, a...);
    };
    header("Running %dD CMAES\nSC: %s\nFC: %s\n", Dimension, d.sc_path.c_str(), d.fc_tril_path.c_str());
    if (d.heterogeneous) header("Maps: %s\n", d.maps_path.c_str());
    header("Free parameters: ");
    for (auto& kv : d.param_mins) header("%s (%f-%f) ", kv.first.c_str(), kv.second, d.param_maxs[kv.first]);
    header("\nFCD step %d, FCD window %d, Simulation random seed %d, CMAES random seed %d, sigma %f, alphacov %f, "
         "gamma_scale %f, bound_soft_edge %f, Variante %d, early stop gens %d, early stop tol %f\n",
         d.window_step, d.window_size, d.rand_seed, d.SeedMW, cp.sigma, cp.alphacov, cp.gamma_scale,
         cp.bound_soft_edge, cp.variante, cp.early_stop_gens, cp.early_stop_tol);

    // plan: configuration, targets, noise
    bnm_config cfg;
    bnm_config_default(&cfg);
    bnm_config_from_env(&cfg);
    cfg.nodes = d.nodes;
    cfg.max_sims = d.lambda;
    cfg.time_steps = d.time_steps;
    cfg.bold_tr = d.BOLD_TR;
    cfg.window_step = d.window_step;
    cfg.window_size = d.window_size;
    cfg.do_fic = d.do_fic;
    cfg.calculate_fic_penalty = d.do_fic;
    cfg.no_fcd = no_fcd;
    cfg.noise_seed = (uint64_t)d.rand_seed;
    const char* pe = std::getenv("BNM_B200_PRECISION");
    if (pe && !std::strcmp(pe, "f64")) cfg.precision = BNM_PREC_F64;
    if (pe && !std::strcmp(pe, "f32ref")) cfg.precision = BNM_PREC_F32_REF;
    // reference-order arithmetic keeps FP64 co-moment FC and the FP32 SIMT FCD
    if (cfg.precision != BNM_PREC_F32) cfg.gram = BNM_GRAM_F32;
    const char* ge = std::getenv("BNM_B200_GRAM");
    if (ge && !std::strcmp(ge, "f32")) cfg.gram = BNM_GRAM_F32;
    if (ge && !std::strcmp(ge, "bf16")) cfg.gram = BNM_GRAM_BF16;
    if (ge && !std::strcmp(ge, "bf16x3")) cfg.gram = BNM_GRAM_BF16_SPLIT;
    const char* ne = std::getenv("BNM_B200_NOISE");
    const bool philox = ne && !std::strcmp(ne, "philox");
    cfg.noise_mode = philox ? BNM_NOISE_PHILOX : BNM_NOISE_HOST;
    bnm_sizes sz;
    if (bnm_config_sizes(&cfg, &sz)) die("configuration");
    std::vector<float> noise;
    auto t0 = std::chrono::high_resolution_clock::now();
    if (!philox) {  // run_CMAES.cpp:640-657
        std::printf("Noise precalculation...\n");
        noise.resize((size_t)sz.noise_len);
        std::mt19937 gen(d.rand_seed);
        std::normal_distribution<float> dist(0, 1);
        for (auto& v : noise) v = dist(gen);
        std::printf("took %lf s\n",
                    std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count());
    }
    bnm_plan* plan = nullptr;
    if (bnm_plan_create(&cfg, sc.data(), emp_fc.data(), (int)emp_fc.size(), no_fcd ? nullptr : emp_fcd.data(),
                        (int)emp_fcd.size(), philox ? nullptr : noise.data(), (int64_t)noise.size(), &plan))
        die("plan");
    noise.clear();
    noise.shrink_to_fit();

    cp.lambda = d.lambda;
    cp.dimension = Dimension;
    cp.seed_mw = d.SeedMW;
    cp.it_max = d.itMax;
    bnm_cmaes* es = nullptr;
    if (resumed) {
        bnm_cmaes_params rp;
        bnm_cmaes_params_of(resumed, &rp);
        if (rp.lambda != cp.lambda || rp.dimension != cp.dimension || rp.seed_mw != cp.seed_mw ||
            rp.it_max != cp.it_max || rp.variante != cp.variante || rp.sigma != cp.sigma) {
            std::fprintf(stderr, "Error: checkpoint %s was written for other CMA-ES settings\n", ckpt.c_str());
            return 1;
        }
        es = resumed;
        std::printf("Resuming from %s at iteration %d\n", ckpt.c_str(), bnm_cmaes_iteration(es));
    } else if (bnm_cmaes_create(&cp, &es)) {
        std::fprintf(stderr, "Error: bad CMA-ES settings\n");
        return 1;
    }
    const char* me = std::getenv("BNM_B200_METRICS");  // JSON-lines sidecar, appended
    FILE* metrics = me ? std::fopen(me, "a") : nullptr;
    if (me && !metrics) {
        std::fprintf(stderr, "Error opening metrics file %s\n", me);
        return 1;
    }
    const char* mg = std::getenv("BNM_B200_MAX_GENERATIONS");
    const int max_gens = mg ? std::atoi(mg) : 0;  // generations of this process (0: no limit)
    int gens_here = 0;
    const int L = d.lambda, N = d.nodes;
    std::vector<double> G(L), wEE((size_t)L * N), wEI((size_t)L * N), wIE((size_t)L * N, 0.0);
    std::vector<double> feas((size_t)Dimension * L), cost(L), pen(L), total(L), penalized(L);
    bnm_batch_out out;
    std::memset(&out, 0, sizeof out);
    out.cost = cost.data();
    out.fic_penalty = pen.data();

    auto params_of = [&](const double* x, int stride, int i) {
        std::map<std::string, double> c = d.params;
        for (size_t f = 0; f < d.free_params.size(); f++)
            c[d.free_params[f]] = d.param_diffs[d.free_params[f]] * x[f * stride + i] + d.param_mins[d.free_params[f]];
        return c;
    };
    int it = bnm_cmaes_iteration(es);
    while (it < d.itMax) {
        both("Iteration %d\n", it);
        bnm_cmaes_samples(es, feas.data(), nullptr, nullptr);
        for (int i = 0; i < L; i++) {
            auto c = params_of(feas.data(), L, i);
            d.calculate_params(c, i, G.data(), wEE.data(), wEI.data(), wIE.data());
        }
        auto t1 = std::chrono::high_resolution_clock::now();
        if (bnm_run(plan, L, G.data(), wEE.data(), wEI.data(), d.do_fic ? nullptr : wIE.data(), &out))
            die("run_simulations");
        const double gen_s = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t1).count();
        std::printf("took %lf s\n", gen_s);
        for (int i = 0; i < L; i++) total[i] = cost[i] + (d.do_fic ? pen[i] : 0.0);
        const int this_it = it;
        const int new_it = bnm_cmaes_tell(es, total.data(), penalized.data());
        if (metrics) {  // one JSON line per generation
            double ms[6];
            bnm_last_timings(plan, ms);
            double bx = 0;
            bnm_cmaes_best(es, nullptr, &bx);
            std::fprintf(metrics,
                         "{\"iteration\": %d, \"simulations\": %d, \"wall_s\": %.6f, \"sims_per_s\": %.4f, "
                         "\"device_ms\": {\"fic\": %.4f, \"integrate\": %.4f, \"fc_window\": %.4f, "
                         "\"fcd_ks\": %.4f, \"gof\": %.4f, \"total\": %.4f}, \"generation_best_cost\": %.9g, "
                         "\"best_gof\": %.9g, \"graph_launch\": %s}\n",
                         this_it, L, gen_s, L / gen_s, ms[0], ms[1], ms[2], ms[3], ms[4], ms[5],
                         *std::min_element(total.begin(), total.end()), bx, [&] {
                             int32_t g = 0;
                             bnm_plan_graph(plan, &g);
                             return g ? "true" : "false";
                         }());
            std::fflush(metrics);
        }
        for (int i = 0; i < L; i++) {
            both("\t IndPar %d: ", i);
            auto c = params_of(feas.data(), L, i);
            for (auto& f : d.free_params) both("%s=%f,", f.c_str(), c[f]);
            if (d.do_fic)
                both("gof=%f,fic_penalty=%f,penalized_cost=%f\n", -total[i] + pen[i], pen[i], penalized[i]);
            else
                both("gof=%f,penalized_cost=%f\n", -total[i], penalized[i]);
        }
        it = new_it;
        if (!ckpt.empty()) {
            std::fflush(log);
            if (!write_checkpoint(ckpt, es, std::ftell(log))) {
                std::fprintf(stderr, "Error: cannot write checkpoint %s\n", ckpt.c_str());
                return 1;
            }
        }
        if (max_gens > 0 && ++gens_here >= max_gens && it < d.itMax) {
            std::printf("Stopped after %d generations at iteration %d%s\n", gens_here, it,
                        ckpt.empty() ? "" : "; rerun with the same checkpoint to continue");
            std::fclose(log);
            if (metrics) std::fclose(metrics);
            bnm_cmaes_destroy(es);
            bnm_plan_destroy(plan);
            return 75;  // EX_TEMPFAIL: incomplete, to be continued
        }
    }

    // best feasible point, rerun and saved (run_CMAES.cpp:821-906, bnm.cu:771-833)
    std::vector<double> best(Dimension);
    double best_val = 0;
    bnm_cmaes_best(es, best.data(), &best_val);
    both("Best feasible parameters: ");
    auto c = params_of(best.data(), 1, 0);
    for (auto& f : d.free_params) both("%s=%f,", f.c_str(), c[f]);
    d.calculate_params(c, 0, G.data(), wEE.data(), wEI.data(), wIE.data());
    std::vector<double> bold((size_t)sz.frames * N), ext(6 * (size_t)N), wie_out(N);
    int32_t failed = 0, ntrials = 0;
    bnm_batch_out o1;
    std::memset(&o1, 0, sizeof o1);
    o1.cost = cost.data();
    o1.fic_penalty = pen.data();
    o1.bold = bold.data();
    o1.ext_means = ext.data();
    o1.w_ie = wie_out.data();
    o1.fic_failed = &failed;
    o1.fic_ntrials = &ntrials;
    if (bnm_run(plan, 1, G.data(), wEE.data(), wEI.data(), d.do_fic ? nullptr : wIE.data(), &o1)) die("best rerun");
    {
        FILE* f = std::fopen((sims_prefix + "bold.txt").c_str(), "w");
        for (int i = 0; f && i < sz.frames; i++) {
            for (int j = 0; j < N; j++) std::fprintf(f, "%f ", bold[(size_t)i * N + j]);
            std::fprintf(f, "\n");
        }
        if (f) std::fclose(f);
        const char* names[6] = {"S_E", "I_E", "r_E", "S_I", "I_I", "r_I"};
        for (int v = 0; v < 6; v++) write_row(sims_prefix + names[v] + ".txt", ext.data() + (size_t)v * N, N);
        write_row(sims_prefix + "w_EE.txt", wEE.data(), N);
        write_row(sims_prefix + "w_EI.txt", wEI.data(), N);
        if (d.do_fic) {
            write_row(sims_prefix + "w_IE.txt", wie_out.data(), N);
            if (cfg.numerical_fic) {
                FILE* ff = std::fopen((sims_prefix + "fic_failed.txt").c_str(), "w");
                if (ff) {
                    std::fprintf(ff, "%d", failed);
                    std::fclose(ff);
                }
                FILE* ft = std::fopen((sims_prefix + "fic_ntrials.txt").c_str(), "w");
                if (ft) {
                    std::fprintf(ft, "%d of max %d", ntrials, cfg.max_fic_trials);
                    std::fclose(ft);
                }
            }
        }
    }
    if (d.do_fic)
        both("gof=%f,fic_penalty=%f,gof_fic_penalty=%f\n", -cost[0], pen[0], best_val);
    else
        both("gof=%f\n", best_val);
    if (metrics) std::fclose(metrics);
    std::fclose(log);
    bnm_cmaes_destroy(es);
    bnm_plan_destroy(plan);
    return 0;
}
