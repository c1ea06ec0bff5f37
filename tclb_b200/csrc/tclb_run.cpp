// tclb_run: command-line runner of TCLB case files on the B200 engine.
//
//   tclb_run <model> <case.xml> [--fp64] [--storage same|fp16|fp16s|bf16|bf16s] [--output DIR] [--quiet]
//
// <model> is d2q9, d3q19 or d3q27_cumulant -- TCLB builds one executable per
// model (CLB/<model>/main); here one runner takes the model as its first
// argument.
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/tclb_b200.h"

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s <d2q9|d3q19|d3q27_cumulant> <case.xml> [--fp64] [--storage S] [--output DIR] [--quiet]\n",
                 argv[0]);
    return 2;
  }
  const std::string m = argv[1];
  const int model = m == "d2q9" ? TCLB_MODEL_D2Q9
                    : m == "d3q19" ? TCLB_MODEL_D3Q19
                    : (m == "d3q27_cumulant" || m == "d3q27c") ? TCLB_MODEL_D3Q27_CUMULANT : -1;
  if (model < 0) {
    std::fprintf(stderr, "unknown model %s\n", argv[1]);
    return 2;
  }
  int precision = TCLB_FP32, storage = TCLB_STORAGE_SAME, verbose = 1;
  const char* out = nullptr;
  for (int i = 3; i < argc; i++) {
    const std::string a = argv[i];
    if (a == "--fp64") precision = TCLB_FP64;
    else if (a == "--quiet") verbose = 0;
    else if (a == "--output" && i + 1 < argc) out = argv[++i];
    else if (a == "--storage" && i + 1 < argc) {
      const std::string s = argv[++i];
      storage = s == "fp16" ? TCLB_STORAGE_FP16 : s == "fp16s" ? TCLB_STORAGE_FP16_SHIFT
                : s == "bf16" ? TCLB_STORAGE_BF16 : s == "bf16s" ? TCLB_STORAGE_BF16_SHIFT : TCLB_STORAGE_SAME;
    } else {
      std::fprintf(stderr, "unknown option %s\n", a.c_str());
      return 2;
    }
  }
  const int rc = tclb_case_run(argv[2], model, precision, storage, out, verbose);
  if (rc) {
    std::fprintf(stderr, "tclb_run: %s\n", tclb_case_last_error());
    return 1;
  }
  return 0;
}
