// autotune.h -- the learned cost model's choice of form and split count inside the drop-in
// executables (MGXBENCH_FORM=auto).
//
// The model file is the JSON written by mgxbench_b200.autotune.MlpModel.save: standardisation
// constants (xmean, xstd, ymean, ystd), the flat parameter vector of the 6 -> 64 -> 64 -> 2 MLP
// and the candidate list [[tile, splits], ...].  Inference runs on the GPU through
// mgx_mlp_forward; the rule is the one of mgxbench_b200.autotune.choose: the fastest candidate
// whose predicted normwise error meets the target (with a guard band of 2 for the CRT form), else
// the candidate with the most splits.
// MGXBench's own AUTO mode (autotuning/predictive.py:606-657) chooses a communication library
// from a regression of measured times; here the choice is the kernel configuration.
#pragma once

#include <cuda_runtime.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "mgxgemm.h"

namespace mm {

struct AutoChoice {
    int form = -1;        // MGX_FORM_FP64, MGX_FORM_OZAKI or MGX_FORM_CRT
    int splits = 0;
    int ksplit = 1;       // FP64 split-K slices
    int tile_m = 128;     // FP64 output tile height (64 or 128)
    double predicted_s = 0.0;
    double predicted_err = 0.0;
    std::string model_path;
};

// Numbers of the JSON array stored under "key" (the model file is written by this project, so
// a flat scan for the key and its bracketed list is enough; nested lists are flattened).
inline bool json_numbers(const std::string &text, const char *key, std::vector<double> *out)
{
    const std::string k = std::string("\"") + key + "\"";
    size_t p = text.find(k);
    if (p == std::string::npos) return false;
    p = text.find(':', p + k.size());
    if (p == std::string::npos) return false;
    p = text.find_first_not_of(" \t\r\n", p + 1);
    if (p == std::string::npos || text[p] != '[') return false;
    int depth = 0;
    out->clear();
    const char *s = text.c_str();
    for (size_t i = p; i < text.size(); ++i) {
        const char c = s[i];
        if (c == '[') {
            ++depth;
        } else if (c == ']') {
            if (--depth == 0) return true;
        } else if (c == '-' || c == '+' || c == '.' || (c >= '0' && c <= '9')) {
            char *end = nullptr;
            const double v = strtod(s + i, &end);
            if (end == s + i) return false;
            out->push_back(v);
            i = (size_t)(end - s) - 1;
        }
    }
    return false;
}

// Directory of this executable (for the default model path).
inline std::string exe_dir()
{
    char buf[4096];
    const ssize_t n = readlink("/proc/self/exe", buf, sizeof buf - 1);
    if (n <= 0) return ".";
    buf[n] = '\0';
    std::string p(buf);
    const size_t slash = p.rfind('/');
    return slash == std::string::npos ? std::string(".") : p.substr(0, slash);
}

inline std::string default_model_path() { return exe_dir() + "/../mgxbench_b200/data/mlp_b200.json"; }

// Tile ids of the candidates (mgxbench_b200.autotune): 0, 2, 3, 4, 5 are the FP64 kernel's
// 128 x 128 tiles with the K range cut into 1, 2, 4, 8, 16 slices; 9, 10, 11, 12 its 64 x 128
// tiles with 1, 2, 4, 8 slices and 13 its 64 x 128 tiles in the stream-K schedule (K slices 0);
// 1, 6, 7 are the Ozaki kernel with 1, 4, 16 slices; 8 is the CRT form (its "splits" is the
// modulus count).
inline int tile_ksplit(int tile)
{
    switch (tile) {
    case 2: return 2;
    case 3: return 4;
    case 4: return 8;
    case 5: return 16;
    case 6: return 4;
    case 7: return 16;
    case 10: return 2;
    case 11: return 4;
    case 12: return 8;
    case 13: return 0;  // stream-K
    default: return 1;
    }
}

inline int tile_rows(int tile) { return (tile >= 9 && tile <= 13) ? 64 : 128; }
inline bool tile_is_crt(int tile) { return tile == 8; }
inline bool tile_is_fp64(int tile) { return tile != 1 && tile != 6 && tile != 7 && !tile_is_crt(tile); }

// Same rule as mgxbench_b200.autotune.splitk_applies: each slice gets a 32-wide K block, the
// partial products fit 4 GiB, and an Ozaki split needs K within one int32 accumulation.
inline bool splitk_applies(int m, int n, int k, int ksplit, int splits)
{
    if (ksplit <= 1) return true;  // whole K, or stream-K
    if (splits > 0 && k > mgx_ozaki_kmax(splits)) return false;
    return (k + 31) / 32 >= ksplit && (double)ksplit * m * n * 8.0 <= 4294967296.0;
}

// Loads the model at `path` and picks the form and split count for an m x n x k product whose
// inputs span `exp_range` binades either side of 1.  Returns 0, or a message in *why.
inline int auto_choose(const std::string &path, int m, int n, int k, double exp_range, double target,
                       AutoChoice *out, std::string *why, bool whole_k_only = false)
{
    std::ifstream f(path);
    if (!f) {
        *why = "cannot read cost model " + path;
        return -1;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    if (text.find("\"mgx-mlp-v1\"") == std::string::npos) {
        *why = path + " is not an mgx-mlp-v1 model";
        return -1;
    }
    std::vector<double> xmean, xstd, ymean, ystd, params, cand;
    if (!json_numbers(text, "xmean", &xmean) || !json_numbers(text, "xstd", &xstd) ||
        !json_numbers(text, "ymean", &ymean) || !json_numbers(text, "ystd", &ystd) ||
        !json_numbers(text, "params", &params) || xmean.size() != 6 || xstd.size() != 6 || ymean.size() != 2 ||
        ystd.size() != 2 || (int)params.size() != mgx_mlp_param_count()) {
        *why = path + ": missing or mis-sized model arrays";
        return -1;
    }
    if (!json_numbers(text, "candidates", &cand) || cand.empty() || cand.size() % 2) {
        // default list: FP64 128-row tiles (1..16 K slices) and 64-row tiles (1..8, stream-K), Ozaki 3..9
        // splits with 1, 4, 16 K slices, CRT 9, 11..16 moduli
        cand = {0, 0, 2, 0, 3, 0, 4, 0, 5, 0, 9, 0, 10, 0, 11, 0, 12, 0, 13, 0};
        for (int t : {1, 6, 7})
            for (int s = 3; s <= 9; ++s) {
                cand.push_back(t);
                cand.push_back(s);
            }
        for (int q : {9, 11, 12, 13, 14, 15, 16}) {
            cand.push_back(8);
            cand.push_back(q);
        }
    }
    {   // keep the candidates that apply to this product
        std::vector<double> keep;
        for (size_t c = 0; c + 1 < cand.size(); c += 2) {
            const int ks = tile_ksplit((int)cand[c]);
            if (tile_is_crt((int)cand[c])) {
                if (k > mgx_crt_kmax()) continue;
            } else if (!splitk_applies(m, n, k, ks, (int)cand[c + 1]) || (whole_k_only && ks > 1)) {
                continue;
            }
            keep.push_back(cand[c]);
            keep.push_back(cand[c + 1]);
        }
        cand.swap(keep);
    }
    const int nc = (int)cand.size() / 2;
    if (nc == 0) {
        *why = path + ": no candidate applies to this product";
        return -1;
    }
    std::vector<float> X((size_t)nc * 6), P(params.begin(), params.end()), Y((size_t)nc * 2);
    for (int c = 0; c < nc; ++c) {
        const double feat[6] = {std::log2((double)m), std::log2((double)n), std::log2((double)k), exp_range,
                                cand[2 * c], cand[2 * c + 1]};
        for (int j = 0; j < 6; ++j) X[(size_t)c * 6 + j] = (float)((feat[j] - xmean[j]) / xstd[j]);
    }
    float *dX = nullptr, *dP = nullptr, *dY = nullptr;
    int rc = 0;
    if (cudaMalloc(&dX, X.size() * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&dP, P.size() * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&dY, Y.size() * sizeof(float)) != cudaSuccess ||
        cudaMemcpy(dX, X.data(), X.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dP, P.data(), P.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        *why = "cannot stage the cost model on the device";
        rc = -1;
    }
    if (rc == 0 && mgx_mlp_forward(dX, nc, dP, dY, nullptr) != MGX_SUCCESS) {
        *why = std::string("cost model inference failed: ") + mgx_last_error_message();
        rc = -1;
    }
    if (rc == 0 && cudaMemcpy(Y.data(), dY, Y.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
        *why = "cannot read the cost model's predictions";
        rc = -1;
    }
    cudaFree(dX);
    cudaFree(dP);
    cudaFree(dY);
    if (rc) return rc;
    int best = -1, most = -1;
    double best_t = 0.0;
    for (int c = 0; c < nc; ++c) {
        const double t = std::exp(Y[(size_t)c * 2] * ystd[0] + ymean[0]);
        const double e = std::pow(10.0, Y[(size_t)c * 2 + 1] * ystd[1] + ymean[1]);
        // a CRT candidate needs a guard band of 2 (mgxbench_b200.autotune.CRT_ERROR_MARGIN)
        const double guard = tile_is_crt((int)cand[2 * c]) ? 2.0 : 1.0;
        if (e * guard <= target && (best < 0 || t < best_t)) {
            best = c;
            best_t = t;
        }
        // fallback: most splits, then the lowest tile id (mgxbench_b200.autotune.choose)
        if (most < 0 || cand[2 * c + 1] > cand[2 * most + 1] ||
            (cand[2 * c + 1] == cand[2 * most + 1] && cand[2 * c] < cand[2 * most]))
            most = c;
    }
    const int pick = best >= 0 ? best : most;
    out->form = tile_is_crt((int)cand[2 * pick]) ? MGX_FORM_CRT
                : tile_is_fp64((int)cand[2 * pick]) ? MGX_FORM_FP64 : MGX_FORM_OZAKI;
    out->splits = (int)cand[2 * pick + 1];
    out->ksplit = tile_ksplit((int)cand[2 * pick]);
    out->tile_m = tile_rows((int)cand[2 * pick]);
    out->predicted_s = std::exp(Y[(size_t)pick * 2] * ystd[0] + ymean[0]);
    out->predicted_err = std::pow(10.0, Y[(size_t)pick * 2 + 1] * ystd[1] + ymean[1]);
    out->model_path = path;
    return 0;
}

// Normwise error target of the automatic choice (MGXBENCH_TARGET_ERR, default 1e-15); the
// executables also validate an automatically chosen form against it.
inline double auto_target()
{
    const char *t = getenv("MGXBENCH_TARGET_ERR");
    return (t && *t) ? atof(t) : 1e-15;
}

// MGXBENCH_FORM=auto: replaces *form / *splits / *form_name with the cost model's choice for an
// m x n x k product and prints it.  The model is MGXBENCH_AUTO_MODEL (default
// ../mgxbench_b200/data/mlp_b200.json beside the executable); the target is
// MGXBENCH_TARGET_ERR (normwise, default 1e-15).  Exits with `exit_code` if the model is
// unusable: AUTO without a model is an error, as in MGXBench (autotuning/predictive.py:609-611).
inline void resolve_auto_form(int *form, int *splits, int *ksplit, int *tile_m, std::string *form_name, int m, int n,
                              int k, double exp_range, int exit_code, bool whole_k_only)
{
    if (*form != 2) return;
    const char *env = getenv("MGXBENCH_AUTO_MODEL");
    const std::string path = (env && *env) ? std::string(env) : default_model_path();
    const double target = auto_target();
    AutoChoice c;
    std::string why;
    if (auto_choose(path, m, n, k, exp_range, target, &c, &why, whole_k_only) != 0) {
        fprintf(stderr, "AUTO: %s\n", why.c_str());
        fflush(stderr);
        exit(exit_code);
    }
    *form = c.form == MGX_FORM_OZAKI ? 1 : (c.form == MGX_FORM_CRT ? 3 : 0);
    *splits = c.form == MGX_FORM_FP64 ? 0 : c.splits;
    *ksplit = c.ksplit;
    *tile_m = c.form == MGX_FORM_FP64 ? c.tile_m : 128;
    *form_name = c.form == MGX_FORM_OZAKI ? "ozaki" : (c.form == MGX_FORM_CRT ? "crt" : "fp64");
    printf("mmb autotune: model=%s m=%d n=%d k=%d exp_range=%g target=%.3e choice=%s splits=%d ksplit=%d "
           "tile_m=%d predicted_s=%.6e predicted_err=%.3e\n",
           path.c_str(), m, n, k, exp_range, target, form_name->c_str(), *splits, *ksplit, *tile_m, c.predicted_s,
           c.predicted_err);
}

}  // namespace mm
