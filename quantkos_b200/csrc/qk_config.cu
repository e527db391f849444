// YAML configuration front-end, UInputs validation, and the config-driven run
// (MCDispatcher::launch_montecarlo) with the .paths writer and the payoff
// percentiles.
//
// Reference pieces (paths relative to the reference project):
//   Parser::parse                      src/IO/ConfigParser.cpp:36-294
//   keys / enum names                  include/core/config/ConfigFileKeys.hpp:30-160,
//                                      include/core/config/ConfigFileKeysEnumMaps.hpp:50-192
//   UInputs defaults and validate()    include/core/config/Config.hpp:50-775
//   BinWriter / BinHeader (.paths)     include/IO/IOBinary.hpp:72-249
//   payoff percentiles                 include/core/options/OptionPricer.hpp:340-360
// yaml-cpp is not used: the files are two- or three-level maps of scalars, read
// by the small reader below (comments, quotes, block nesting by indentation).
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "qk_engine.h"
#include "qk_host.h"
#include "qk_kernels.h"

namespace {

using qk::fail;

std::string trim(const std::string &s) {
    size_t b = 0, e = s.size();
    while (b < e && (s[b] == ' ' || s[b] == '\t' || s[b] == '\r')) ++b;
    while (e > b && (s[e - 1] == ' ' || s[e - 1] == '\t' || s[e - 1] == '\r')) --e;
    return s.substr(b, e - b);
}

std::string strip_comment(const std::string &line) {
    bool sq = false, dq = false;
    for (size_t i = 0; i < line.size(); ++i) {
        const char ch = line[i];
        if (ch == '\'' && !dq) sq = !sq;
        else if (ch == '"' && !sq) dq = !dq;
        else if (ch == '#' && !sq && !dq && (i == 0 || line[i - 1] == ' ' || line[i - 1] == '\t')) return line.substr(0, i);
    }
    return line;
}

std::string unquote(const std::string &v) {
    if (v.size() >= 2 && ((v.front() == '"' && v.back() == '"') || (v.front() == '\'' && v.back() == '\'')))
        return v.substr(1, v.size() - 2);
    return v;
}

// Flattened YAML map: "Block.Key" -> scalar text; blocks (keys without a value) are
// recorded with an empty value and present = true.
struct YamlDoc {
    std::map<std::string, std::string> values;
    std::map<std::string, bool> blocks;
};

qk_status parse_yaml(const std::string &text, YamlDoc &doc) {
    std::istringstream in(text);
    std::string raw;
    std::vector<std::pair<int, std::string>> stack;  // (indent, key)
    int lineno = 0;
    while (std::getline(in, raw)) {
        ++lineno;
        const std::string line = strip_comment(raw);
        if (trim(line).empty()) continue;
        if (trim(line) == "---") continue;
        int indent = 0;
        while (indent < static_cast<int>(line.size()) && (line[indent] == ' ' || line[indent] == '\t')) ++indent;
        const std::string body = trim(line);
        size_t colon = std::string::npos;
        bool sq = false, dq = false;
        for (size_t i = 0; i < body.size(); ++i) {
            const char ch = body[i];
            if (ch == '\'' && !dq) sq = !sq;
            else if (ch == '"' && !sq) dq = !dq;
            else if (ch == ':' && !sq && !dq && (i + 1 == body.size() || body[i + 1] == ' ' || body[i + 1] == '\t')) {
                colon = i;
                break;
            }
        }
        if (colon == std::string::npos)
            return fail(QK_ERR_PARSE, "Config Error: Invalid YAML syntax -> line " + std::to_string(lineno) + ": '" + body + "'");
        const std::string key = trim(body.substr(0, colon));
        const std::string val = trim(body.substr(colon + 1));
        if (key.empty()) return fail(QK_ERR_PARSE, "Config Error: Invalid YAML syntax -> empty key at line " + std::to_string(lineno));
        while (!stack.empty() && stack.back().first >= indent) stack.pop_back();
        std::string path;
        for (const auto &s : stack) path += s.second + ".";
        path += key;
        if (val.empty()) {
            doc.blocks[path] = true;
            stack.emplace_back(indent, key);
        } else {
            doc.values[path] = unquote(val);
        }
    }
    return QK_OK;
}

bool has(const YamlDoc &d, const std::string &k) { return d.values.count(k) > 0; }

qk_status get_real(const YamlDoc &d, const std::string &k, double *out) {
    auto it = d.values.find(k);
    if (it == d.values.end()) return QK_OK;
    const char *s = it->second.c_str();
    char *end = nullptr;
    errno = 0;
    const double v = std::strtod(s, &end);
    if (end == s || *end != '\0' || errno == ERANGE)
        return fail(QK_ERR_PARSE, "Config Error: bad conversion of '" + it->second + "' to a number for " + k);
    *out = v;
    return QK_OK;
}

template <class I>
qk_status get_int(const YamlDoc &d, const std::string &k, I *out) {
    auto it = d.values.find(k);
    if (it == d.values.end()) return QK_OK;
    const char *s = it->second.c_str();
    char *end = nullptr;
    errno = 0;
    long long v;
    if (std::is_unsigned<I>::value) v = static_cast<long long>(std::strtoull(s, &end, 10));
    else v = std::strtoll(s, &end, 10);
    if (end == s || *end != '\0' || errno == ERANGE)
        return fail(QK_ERR_PARSE, "Config Error: bad conversion of '" + it->second + "' to an integer for " + k);
    *out = static_cast<I>(v);
    return QK_OK;
}

qk_status get_bool(const YamlDoc &d, const std::string &k, int32_t *out) {
    auto it = d.values.find(k);
    if (it == d.values.end()) return QK_OK;
    std::string v = it->second;
    std::transform(v.begin(), v.end(), v.begin(), [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
    if (v == "true" || v == "yes" || v == "on" || v == "y" || v == "1") *out = 1;
    else if (v == "false" || v == "no" || v == "off" || v == "n" || v == "0") *out = 0;
    else return fail(QK_ERR_PARSE, "[" + k + "] must be a boolean value (true/false, yes/no, 1/0).");
    return QK_OK;
}

qk_status get_enum(const YamlDoc &d, const std::string &k, const std::vector<std::pair<std::string, int>> &m,
                   int32_t *out) {
    auto it = d.values.find(k);
    if (it == d.values.end()) return QK_OK;
    for (const auto &p : m)
        if (p.first == it->second) {
            *out = p.second;
            return QK_OK;
        }
    // StrEnumMap iterates a std::map, so allowed names are listed in sorted order (ConfigFileKeysEnumMaps.hpp:176-190)
    std::vector<std::string> names;
    for (const auto &p : m) names.push_back(p.first);
    std::sort(names.begin(), names.end());
    std::string err = "Config Error: Invalid value '" + it->second + "' for " + k + ".\nAllowed options: [ ";
    for (const auto &n : names) err += n + " ";
    err += "]";
    return fail(QK_ERR_PARSE, err);
}

const std::vector<std::pair<std::string, int>> kOptTypes = {
    {"European", QK_EUROPEAN}, {"Asian", QK_ASIAN}, {"BarrierUpAndOut", QK_BARRIER_UP_OUT},
    {"BarrierDownAndOut", QK_BARRIER_DOWN_OUT}, {"BarrierUpAndIn", QK_BARRIER_UP_IN},
    {"BarrierDownAndIn", QK_BARRIER_DOWN_IN}, {"LookbackFloatingStrike", QK_LOOKBACK_FLOATING},
    {"LookbackFixedStrike", QK_LOOKBACK_FIXED}, {"BinaryCashOrNothing", QK_BINARY_CASH},
    {"BinaryAssetOrNothing", QK_BINARY_ASSET}, {"American", QK_AMERICAN}};
const std::vector<std::pair<std::string, int>> kRights = {{"Call", QK_CALL}, {"Put", QK_PUT}};
const std::vector<std::pair<std::string, int>> kSchemes = {
    {"Euler", QK_EULER}, {"ImplicitMilstein", QK_IMPLICIT_MILSTEIN}, {"AndersonQE", QK_ANDERSEN_QE}};
const std::vector<std::pair<std::string, int>> kFormats = {{"BIN", 0}, {"TXT", 1}};
const std::vector<std::pair<std::string, int>> kVerbosity = {{"None", 0}, {"Low", 1}, {"Medium", 2}, {"High", 3}};
const std::vector<std::pair<std::string, int>> kPrecisions = {{"FP64", QK_FP64}, {"FP32", QK_FP32}};
const std::vector<std::pair<std::string, int>> kEngines = {{"plain", 0}, {"batch", 1}};
const std::vector<std::pair<std::string, int>> kBases = {{"Laguerre3", QK_LSM_LAGUERRE3}, {"PolySV", QK_LSM_POLY_SV}};

#define QK_TRY(x)                         \
    do {                                  \
        const qk_status s_ = (x);         \
        if (s_ != QK_OK) return s_;       \
    } while (0)

void copy_str(char *dst, const std::string &s) {
    std::strncpy(dst, s.c_str(), 255);
    dst[255] = '\0';
}

qk_status fill_config(const YamlDoc &d, qk_config *c) {
    // 3. Market (mandatory)
    if (!d.blocks.count("Market")) return fail(QK_ERR_PARSE, "Config Error: Mandatory block 'Market' missing.");
    QK_TRY(get_real(d, "Market.Price", &c->S0));
    QK_TRY(get_real(d, "Market.Variance", &c->v0));
    QK_TRY(get_real(d, "Market.r", &c->r));
    QK_TRY(get_real(d, "Market.q", &c->q));
    // 4. Options (mandatory)
    if (!d.blocks.count("Options")) return fail(QK_ERR_PARSE, "Config Error: Mandatory block 'Options' missing.");
    QK_TRY(get_enum(d, "Options.OptionType", kOptTypes, &c->opt_type));
    QK_TRY(get_enum(d, "Options.OptionRight", kRights, &c->opt_right));
    QK_TRY(get_real(d, "Options.StrikePrice", &c->K));
    QK_TRY(get_real(d, "Options.BarrierPrice", &c->B));
    // 5. Model (mandatory; exactly one of Heston / Bates)
    if (!d.blocks.count("Model")) return fail(QK_ERR_PARSE, "Config Error: Mandatory block 'Model' missing.");
    auto present = [&](const std::string &b) {
        if (d.blocks.count(b)) return true;
        const std::string pre = b + ".";
        for (const auto &kv : d.values)
            if (kv.first.compare(0, pre.size(), pre) == 0) return true;
        return false;
    };
    const bool has_h = present("Model.Heston"), has_b = present("Model.Bates");
    if (has_h && has_b) return fail(QK_ERR_PARSE, "Config Error: Cannot define both Heston and Bates models simultaneously.");
    if (has_h) {
        c->model = QK_HESTON;
        QK_TRY(get_real(d, "Model.Heston.k", &c->heston_k));
        QK_TRY(get_real(d, "Model.Heston.theta", &c->heston_theta));
        QK_TRY(get_real(d, "Model.Heston.sigma", &c->heston_sigma));
        QK_TRY(get_real(d, "Model.Heston.rho", &c->heston_rho));
    } else if (has_b) {
        c->model = QK_BATES;
        QK_TRY(get_real(d, "Model.Bates.k", &c->bates_k));
        QK_TRY(get_real(d, "Model.Bates.theta", &c->bates_theta));
        QK_TRY(get_real(d, "Model.Bates.sigma", &c->bates_sigma));
        QK_TRY(get_real(d, "Model.Bates.rho", &c->bates_rho));
        QK_TRY(get_real(d, "Model.Bates.lambda_J", &c->bates_lambda));
        QK_TRY(get_real(d, "Model.Bates.mu_J", &c->bates_mu));
        QK_TRY(get_real(d, "Model.Bates.sigma_J", &c->bates_sigma_j));
    } else {
        return fail(QK_ERR_PARSE, "Config Error: Mandatory block 'Model' has requested a non implemented model!");
    }
    // 6. Numerics (optional)
    QK_TRY(get_enum(d, "Numerics.Scheme", kSchemes, &c->scheme));
    // 7. Time (mandatory)
    if (!d.blocks.count("Time")) return fail(QK_ERR_PARSE, "Config Error: Mandatory block 'Time' missing.");
    QK_TRY(get_real(d, "Time.T_End", &c->t_end));
    QK_TRY(get_real(d, "Time.Inp_DT", &c->inp_dt));
    // 8. MC (mandatory)
    if (!d.blocks.count("MC")) return fail(QK_ERR_PARSE, "Config Error: Mandatory block 'MC' missing.");
    QK_TRY(get_bool(d, "MC.Normalize_prices", &c->normalize));
    QK_TRY(get_int(d, "MC.N_Paths", &c->n_paths));
    QK_TRY(get_int(d, "MC.Batch_Size", &c->batch_size));
    QK_TRY(get_int(d, "MC.RNG_Seed", &c->seed));
    QK_TRY(get_int(d, "MC.Max_VRAM_MB", &c->max_vram_mb));
    QK_TRY(get_int(d, "MC.Max_CPU_RAM_MB", &c->max_cpu_ram_mb));
    QK_TRY(get_bool(d, "MC.analyze_risk_neutral_payoff_distribution", &c->analyze_distribution));
    const char *greek_keys[5] = {"MC.compute_delta_et_gamma", "MC.compute_vega_et_vomma", "MC.compute_vanna",
                                 "MC.compute_rho", "MC.compute_theta"};
    const int greek_bits[5] = {QK_GREEK_DELTA_GAMMA, QK_GREEK_VEGA_VOMMA, QK_GREEK_VANNA, QK_GREEK_RHO, QK_GREEK_THETA};
    for (int i = 0; i < 5; ++i) {
        int32_t on = (c->greeks_mask & greek_bits[i]) ? 1 : 0;
        QK_TRY(get_bool(d, greek_keys[i], &on));
        c->greeks_mask = on ? (c->greeks_mask | greek_bits[i]) : (c->greeks_mask & ~greek_bits[i]);
    }
    QK_TRY(get_real(d, "MC.spot_price_relative_bump_size", &c->bump_S_rel));
    QK_TRY(get_real(d, "MC.volatility_absolute_bump_size", &c->bump_vol_abs));
    QK_TRY(get_real(d, "MC.risk_free_rate_absolute_bump_size", &c->bump_r_abs));
    QK_TRY(get_real(d, "MC.time_absolute_bump_size", &c->bump_T_abs));
    // engine extensions (unknown to the reference, which ignores unknown keys)
    QK_TRY(get_enum(d, "MC.Precision", kPrecisions, &c->precision));
    QK_TRY(get_enum(d, "MC.Engine", kEngines, &c->engine));
    QK_TRY(get_enum(d, "MC.LSM_Basis", kBases, &c->lsm_basis));
    QK_TRY(get_int(d, "MC.LSM_Dates", &c->lsm_dates));
    QK_TRY(get_int(d, "MC.Vega_Mode", &c->vega_mode));
    QK_TRY(get_int(d, "MC.Stream", &c->stream));
    QK_TRY(get_bool(d, "MC.Antithetic", &c->antithetic));
    // 9. Output (optional)
    QK_TRY(get_enum(d, "Output.Verbosity", kVerbosity, &c->verbosity));
    if (has(d, "Output.out_dir")) copy_str(c->out_dir, d.values.at("Output.out_dir"));
    if (has(d, "Output.Name_Paths_Out_File")) copy_str(c->paths_file, d.values.at("Output.Name_Paths_Out_File"));
    if (has(d, "Output.Name_Log_File")) copy_str(c->log_file, d.values.at("Output.Name_Log_File"));
    QK_TRY(get_enum(d, "Output.Format", kFormats, &c->format));
    return QK_OK;
}

// .paths header (IOBinary.hpp:72-81): magic, version, bytes per value, paths, steps, dt, scale.
template <class R>
struct BinHeader {
    char key[8] = {'Q', 'U', 'A', 'N', 'T', 'K', 'O', 'S'};
    int32_t version = 1;
    int32_t byte_precision = sizeof(R);
    int32_t total_n_sims = 0;
    int32_t n_time_steps = 0;
    R dt = 0;
    double scale_factor = 1.0;
};

// Paths per stored batch of the .paths output, as MCConfig sizes the reference's
// path batches (PathsMCBatchMem.hpp:330-390): Batch_Size > 0 fixed, -1 all paths,
// 0 automatic from the device budget Max_VRAM_MB / (steps x element size), in
// multiples of 32.  Pricing itself stores no paths.
int64_t stored_batch_paths(const qk_config &cfg, const qk_contract &c) {
    if (cfg.batch_size > 0) return std::min<int64_t>(cfg.batch_size, c.n_paths);
    if (cfg.batch_size == -1) return c.n_paths;
    const double esz = c.precision == QK_FP32 ? 4.0 : 8.0;
    const int64_t fit = static_cast<int64_t>(static_cast<double>(cfg.max_vram_mb) * 1024.0 * 1024.0 /
                                             (static_cast<double>(c.n_steps) * esz));
    return std::min<int64_t>(c.n_paths, std::max<int64_t>(32, fit / 32 * 32));
}

template <class R>
void write_paths_header(std::ofstream &f, int64_t n_paths, int n_steps, double dt, double scale) {
    BinHeader<R> hd;
    hd.total_n_sims = static_cast<int32_t>(n_paths);
    hd.n_time_steps = n_steps;
    hd.dt = static_cast<R>(dt);
    hd.scale_factor = scale;
    f.write(reinterpret_cast<const char *>(&hd), sizeof(hd));
}

// Rows of `count` paths x n_steps spot values in real units, stored normalised.
template <class R>
void write_paths_rows(std::ofstream &f, const double *S, int64_t count, int n_steps, double scale, std::vector<R> &row) {
    row.resize(static_cast<size_t>(count) * n_steps);
    for (size_t i = 0; i < row.size(); ++i) row[i] = static_cast<R>(S[i] / scale);  // payload holds normalised prices
    f.write(reinterpret_cast<const char *>(row.data()), static_cast<std::streamsize>(row.size() * sizeof(R)));
}

template <class R>
qk_status write_paths_file(qk_handle *h, const qk_contract &c, double dt, double scale, const std::string &path,
                           int64_t chunk) {
    std::ofstream f(path, std::ios::out | std::ios::binary);
    if (!f.is_open()) return fail(QK_ERR_INVALID_ARG, "[BinWriter Error] Failed to open binary output file: " + path);
    write_paths_header<R>(f, c.n_paths, c.n_steps, dt, scale);
    std::vector<double> S;
    std::vector<R> row;
    for (int64_t first = 0; first < c.n_paths; first += chunk) {
        const int64_t cnt = std::min(chunk, c.n_paths - first);
        S.resize(static_cast<size_t>(cnt) * c.n_steps);
        const qk_status st = qk_paths_dump(h, &c, first, cnt, S.data(), nullptr);
        if (st != QK_OK) return st;
        write_paths_rows<R>(f, S.data(), cnt, c.n_steps, scale, row);
    }
    if (!f.good()) return fail(QK_ERR_INVALID_ARG, "[BinWriter Error] write failed: " + path);
    return QK_OK;
}

}  // namespace

extern "C" {

qk_status qk_paths_write(const char *path, int32_t precision, int64_t n_paths, int32_t n_steps, double dt,
                         double scale, const double *S) {
    if (!path || !S || n_paths < 1 || n_steps < 1 || !(scale > 0.0))
        return fail(QK_ERR_INVALID_ARG, "qk_paths_write: invalid arguments");
    std::ofstream f(path, std::ios::out | std::ios::binary);
    if (!f.is_open()) return fail(QK_ERR_INVALID_ARG, std::string("[BinWriter Error] Failed to open binary output file: ") + path);
    if (precision == QK_FP32) {
        std::vector<float> row;
        write_paths_header<float>(f, n_paths, n_steps, dt, scale);
        write_paths_rows<float>(f, S, n_paths, n_steps, scale, row);
    } else {
        std::vector<double> row;
        write_paths_header<double>(f, n_paths, n_steps, dt, scale);
        write_paths_rows<double>(f, S, n_paths, n_steps, scale, row);
    }
    if (!f.good()) return fail(QK_ERR_INVALID_ARG, std::string("[BinWriter Error] write failed: ") + path);
    return QK_OK;
}

qk_status qk_config_default(qk_config *c) {
    if (!c) return fail(QK_ERR_INVALID_ARG, "NULL argument");
    std::memset(c, 0, sizeof(*c));
    c->S0 = 100.0;
    c->v0 = 1.0;
    c->r = 0.05;
    c->q = 0.0;
    c->opt_type = QK_EUROPEAN;
    c->opt_right = QK_CALL;
    c->K = 100.0;
    c->B = 100.0;
    c->model = QK_HESTON;
    c->heston_k = c->bates_k = 2.0;
    c->heston_theta = c->bates_theta = 0.04;
    c->heston_sigma = c->bates_sigma = 0.3;
    c->heston_rho = c->bates_rho = -0.7;
    c->bates_lambda = 0.1;
    c->bates_mu = -0.1;
    c->bates_sigma_j = 0.15;
    c->scheme = QK_EULER;
    c->t_end = 1.0;
    c->inp_dt = 0.2;
    c->normalize = 1;
    c->n_paths = 1000;
    c->batch_size = 0;
    c->seed = 184467440737095ULL;
    c->max_vram_mb = 256;
    c->max_cpu_ram_mb = 4000;
    c->bump_S_rel = 0.001;
    c->bump_vol_abs = 0.01;
    c->bump_r_abs = 0.0001;
    c->bump_T_abs = 1.0 / 365.0;
    c->verbosity = 3;
    c->format = 0;
    copy_str(c->out_dir, "outputs");
    copy_str(c->paths_file, "QuantKos.paths");
    copy_str(c->log_file, "QuantKos.log");
    c->precision = QK_FP64;
    c->engine = 0;
    c->lsm_basis = QK_LSM_LAGUERRE3;
    c->lsm_dates = 0;
    c->vega_mode = 0;
    c->stream = 0;
    c->antithetic = 0;
    return QK_OK;
}

qk_status qk_config_validate(qk_config *c) {
    if (!c) return fail(QK_ERR_INVALID_ARG, "NULL argument");
    // MarketConfig / OptionsConfig / MathModelConfig via the contract validator, TimeConfig here
    if (!(c->t_end > 0.0)) return fail(QK_ERR_INVALID_ARG, "[Time.T_End] must be positive.");
    if (!(c->inp_dt > 0.0)) return fail(QK_ERR_INVALID_ARG, "[Time.DT] must be positive.");
    if (c->inp_dt > c->t_end) return fail(QK_ERR_INVALID_ARG, "[Time.DT] must be smaller that total time.");
    c->n_steps = static_cast<int32_t>(std::ceil(c->t_end / c->inp_dt));  // TimeConfig::validate (Config.hpp:359-363)
    c->dt = c->t_end / c->n_steps;
    if (c->batch_size < -1)
        return fail(QK_ERR_INVALID_ARG, "[MC.Batch_Size] Must be a positive integer if you want to impose it, -1 if you want it equal to the max number of paths, and 0 if you want to let the machine handle this.");
    if (c->batch_size > c->n_paths)
        return fail(QK_ERR_INVALID_ARG, "[MC.Batch_Size] The batch size must be smaller that the notal number of realizations.");
    if (c->max_vram_mb <= 0) return fail(QK_ERR_INVALID_ARG, "[MC.Max_VRAM_MB] must be a positive integer.");
    if (c->max_cpu_ram_mb <= 0) return fail(QK_ERR_INVALID_ARG, "[MC.Max_CPU_RAM_MB] must be a positive integer.");
    if (c->format != 0)
        return fail(QK_ERR_INVALID_ARG, "[Configuration Error] Unsupported output format requested. Currently, only the BIN (Binary) writer is fully implemented and supported.");
    qk_contract k;
    qk_greeks g;
    QK_TRY(qk_config_to_contract(c, &k, &g));
    QK_TRY(qk_validate(&k, &g));
    if (c->out_dir[0] != '\0') {
        std::error_code ec;
        std::filesystem::create_directories(c->out_dir, ec);
        if (ec)
            return fail(QK_ERR_INVALID_ARG, std::string("[Configuration Error] The assigned output directory '") + c->out_dir +
                                                "' could not be prepared or accessed.\nDetails: " + ec.message());
    }
    return QK_OK;
}

qk_status qk_config_parse_string(const char *yaml, qk_config *out) {
    if (!yaml || !out) return fail(QK_ERR_INVALID_ARG, "NULL argument");
    qk_config_default(out);
    YamlDoc doc;
    QK_TRY(parse_yaml(yaml, doc));
    QK_TRY(fill_config(doc, out));
    return qk_config_validate(out);
}

qk_status qk_config_parse_file(const char *path, qk_config *out) {
    if (!path || !out) return fail(QK_ERR_INVALID_ARG, "NULL argument");
    if (!std::filesystem::exists(path)) return fail(QK_ERR_PARSE, std::string("Config Error: File not found -> ") + path);
    std::ifstream f(path);
    std::stringstream ss;
    ss << f.rdbuf();
    return qk_config_parse_string(ss.str().c_str(), out);
}

qk_status qk_config_to_contract(const qk_config *c, qk_contract *k, qk_greeks *g) {
    if (!c || !k) return fail(QK_ERR_INVALID_ARG, "NULL argument");
    std::memset(k, 0, sizeof(*k));
    k->S0 = c->S0;
    k->v0 = c->v0;
    k->r = c->r;
    k->q = c->q;
    k->model = c->model;
    k->scheme = c->scheme;
    const bool bates = c->model == QK_BATES;
    k->kappa = bates ? c->bates_k : c->heston_k;
    k->theta = bates ? c->bates_theta : c->heston_theta;
    k->sigma = bates ? c->bates_sigma : c->heston_sigma;
    k->rho = bates ? c->bates_rho : c->heston_rho;
    k->lambda_j = bates ? c->bates_lambda : 0.0;
    k->mu_j = bates ? c->bates_mu : 0.0;
    k->sigma_j = bates ? c->bates_sigma_j : 0.0;
    k->psi_c = 1.5;
    k->T = c->t_end;
    k->n_steps = c->n_steps > 0 ? c->n_steps : static_cast<int32_t>(std::ceil(c->t_end / c->inp_dt));
    k->normalize = c->normalize;
    k->n_paths = c->n_paths;
    k->seed = c->seed;
    k->stream = c->stream;
    k->antithetic = c->antithetic;
    k->precision = c->precision;
    k->n_payoffs = 1;
    k->payoffs[0].type = c->opt_type;
    k->payoffs[0].right = c->opt_right;
    k->payoffs[0].strike = c->K;
    k->payoffs[0].barrier = c->B;
    k->lsm_basis = c->lsm_basis;
    k->lsm_dates = c->lsm_dates;
    if (g) {
        std::memset(g, 0, sizeof(*g));
        g->mask = c->greeks_mask;
        g->vega_mode = c->vega_mode;
        g->bump_S_rel = c->bump_S_rel;
        g->bump_vol = c->bump_vol_abs;
        g->bump_r_abs = c->bump_r_abs;
        g->bump_T_abs = c->bump_T_abs;
    }
    return QK_OK;
}

qk_status qk_run_config(qk_handle *h, const qk_config *cfg, qk_result *out, double *pct) {
    if (!h || !cfg || !out) return fail(QK_ERR_INVALID_ARG, "NULL argument");
    qk_config c = *cfg;
    QK_TRY(qk_config_validate(&c));
    qk_contract k;
    qk_greeks g;
    QK_TRY(qk_config_to_contract(&c, &k, &g));
    if (c.engine == 0) {
        QK_TRY(qk_price_plain(h, &k, g.mask ? &g : nullptr, out));
    } else {
        QK_TRY(qk_price_batch(h, &k, 1, g.mask ? &g : nullptr, out));
    }
    const double scale = k.normalize ? k.S0 : 1.0;
    if (c.paths_file[0] != '\0') {
        const std::string path = (std::filesystem::path(c.out_dir) / c.paths_file).string();
        qk_timing keep;
        qk_last_timing(h, &keep);
        const int64_t chunk = stored_batch_paths(c, k);
        qk_status st = (k.precision == QK_FP32) ? write_paths_file<float>(h, k, c.dt, scale, path, chunk)
                                                : write_paths_file<double>(h, k, c.dt, scale, path, chunk);
        h->timing = keep;
        if (st != QK_OK) return st;
    }
    if (c.analyze_distribution && pct && k.payoffs[0].type != QK_AMERICAN) {
        // OptionPricer::analyze_risk_neutral_discounted_payoff_distribution: sort all payoffs,
        // read 15 order statistics, apply discount and scale.
        std::vector<double> pay;
        QK_TRY(qk::payoffs_dump(h, k, pay));
        std::sort(pay.begin(), pay.end());
        const double N = static_cast<double>(pay.size());
        const double eff = std::exp(-k.r * k.T) * ((k.payoffs[0].type == QK_BINARY_CASH) ? 1.0 : scale);
        const double fr[13] = {0.01, 0.05, 0.10, 0.20, 0.30, 0.40, 0.50, 0.60, 0.70, 0.80, 0.90, 0.95, 0.99};
        pct[0] = pay.front() * eff;
        for (int i = 0; i < 13; ++i) pct[i + 1] = pay[static_cast<size_t>(N * fr[i])] * eff;
        pct[14] = pay.back() * eff;
    }
    return QK_OK;
}

}  // extern "C"
