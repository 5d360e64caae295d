// vfb_cli.cpp -- the `vfb <json_file> <max_formula_size>` command.
//
// Drop-in for the reference's ltl_nocache program (main ltl_nocache.cu:448-487,
// limits of LTL() ltl_nocache.cu:326-348): same positional arguments, same
// stdout line "<json_file>, <formula>" (or "<json_file>, Not found !"), same
// error texts on stderr and exit code 0 on argument errors.  Progress lines go
// to stderr.  Extra options may follow the two positional arguments:
//   --rlx-type N   relaxed-uniqueness rule 1|2|3 when trace bits exceed 126 (default 3)
//   --device N     CUDA device ordinal
//   --mem-gb X     device memory budget in GiB
//   --stats        per-size unique/candidate counts as one JSON line on stderr
//   --quiet        no progress lines
//   --strict-exit  non-zero exit status on errors and when nothing is found
//   --nocache      cache-free search in formula-number order (the reference's
//                  ltl_nocache method) instead of the cached search
//   --bs-max N     when nothing is found up to max size, the BS stage of LTL_BS
//                  (~ & | over the cached formulas' step-0 vectors) up to size N
//   --costs c1,c2,c3,c4,c5,c6,c7,c8
//                  LTL_BS's operator costs (p ~ & | X F G U); the max size is then
//                  the largest cost searched
//   --neg-type N   1: ~ of any formula (default); 2: ~ of propositions only
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/vfb.h"

static void usage(const char* prog) {
  std::fprintf(stderr, "Arguments should be in the form of\n");
  std::fprintf(stderr, "-----------------------------------------------------------------\n");
  std::fprintf(stderr, "%s <input_file_address> <maxLen>\n", prog);
  std::fprintf(stderr, "-----------------------------------------------------------------\n");
}

int main(int argc, char** argv) {
  std::vector<const char*> pos;
  int rlx = 3, device = 0, stats = 0, quiet = 0, strict = 0, nocache = 0, bs_max = 0, neg_type = 1;
  int costs[8] = {1, 1, 1, 1, 1, 1, 1, 1};
  bool weighted = false;
  double mem_gb = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--rlx-type" && i + 1 < argc) rlx = std::atoi(argv[++i]);
    else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
    else if (a == "--mem-gb" && i + 1 < argc) mem_gb = std::atof(argv[++i]);
    else if (a == "--stats") stats = 1;
    else if (a == "--quiet") quiet = 1;
    else if (a == "--strict-exit") strict = 1;
    else if (a == "--nocache") nocache = 1;
    else if (a == "--bs-max" && i + 1 < argc) bs_max = std::atoi(argv[++i]);
    else if (a == "--neg-type" && i + 1 < argc) { neg_type = std::atoi(argv[++i]); weighted = true; }
    else if (a == "--costs" && i + 1 < argc) {
      const std::string v = argv[++i];
      size_t p0 = 0;
      for (int c = 0; c < 8; ++c) {
        const size_t p1 = v.find(',', p0);
        costs[c] = std::atoi(v.substr(p0, p1 == std::string::npos ? std::string::npos : p1 - p0).c_str());
        if (p1 == std::string::npos) break;
        p0 = p1 + 1;
      }
      weighted = true;
    }
    else pos.push_back(argv[i]);
  }
  if (pos.size() != 2) {
    usage(argv[0]);
    return strict ? 2 : 0;
  }
  const int maxLen = std::atoi(pos[1]);
  if (maxLen < 1 || maxLen > 50) {
    std::fprintf(stderr, "Argument maxLen = %s should be between 1 and %d", pos[1], VFB_MAX_SIZE);
    return strict ? 2 : 0;
  }
  if (rlx < 1 || rlx > 3) {
    std::fprintf(stderr, "--rlx-type must be 1, 2 or 3\n");
    return strict ? 2 : 0;
  }
  const std::string file = pos[0];
  char err[512] = {0};
  vfb_json_problem* jp = nullptr;
  if (vfb_read_json(file.c_str(), &jp, err, sizeof(err)) != VFB_OK) {
    std::fprintf(stderr, "%s\n", err);
    return strict ? 2 : 0;
  }
  // limits, with the reference's messages (ltl_nocache.cu:326-348)
  const char* limit = nullptr;
  char msg[160];
  if (maxLen > VFB_MAX_SIZE) {
    std::snprintf(msg, sizeof(msg), "This version supports formulas of size at most %d.\n", VFB_MAX_SIZE);
    limit = msg;
  } else if (jp->inst.num_traces > VFB_MAX_TRACES) {
    std::snprintf(msg, sizeof(msg), "This version supports at most %d samples.\n", VFB_MAX_TRACES);
    limit = msg;
  } else if (jp->inst.num_vars > VFB_MAX_VARS) {
    std::snprintf(msg, sizeof(msg), "This version supports at most %d variables.\n", VFB_MAX_VARS);
    limit = msg;
  } else if (jp->max_length_traces > VFB_MAX_LENGTH) {
    std::snprintf(msg, sizeof(msg), "This version supports traces of size at most %d.\n", VFB_MAX_LENGTH);
    limit = msg;
  }
  if (limit) {
    std::fputs(limit, stderr);
    vfb_json_free(jp);
    return strict ? 2 : 0;
  }
  vfb_opts opts{};
  opts.device = device;
  opts.mem_limit_bytes = (size_t)(mem_gb * (double)(1ULL << 30));
  opts.verbose = quiet ? 0 : 1;
  void* ctx = nullptr;
  vfb_status s = vfb_create(&ctx, &opts);
  if (s != VFB_OK) {
    std::fprintf(stderr, "vfb: cannot initialise the GPU engine: %s\n", vfb_status_str(s));
    vfb_json_free(jp);
    return 3;
  }
  vfb_instance inst = jp->inst;
  inst.max_size = maxLen;
  inst.rlx_type = rlx;
  vfb_result res;
  if (nocache) s = vfb_solve_exhaustive(ctx, &inst, &res);
  else if (weighted) s = vfb_solve_costs(ctx, &inst, costs, neg_type, &res);
  else if (bs_max > maxLen) s = vfb_solve_bs(ctx, &inst, bs_max, &res);
  else s = vfb_solve(ctx, &inst, &res);
  int rc = 0;
  if (res.status == VFB_OK) {
    const int n = vfb_format_infix(&res, jp->names, nullptr, 0);
    std::string text(n > 0 ? (size_t)n + 1 : 1, '\0');
    vfb_format_infix(&res, jp->names, &text[0], text.size());
    text.resize(n > 0 ? (size_t)n : 0);
    std::printf("%s, %s\n", file.c_str(), text.c_str());
  } else if (res.status == VFB_NOT_FOUND) {
    std::printf("%s, %s\n", file.c_str(), "Not found !");
    rc = strict ? 1 : 0;
  } else {
    std::fprintf(stderr, "vfb: %s\n", vfb_status_str(res.status));
    rc = strict ? 3 : 0;
  }
  if (stats) {
    std::fprintf(stderr, "{\"status\": \"%s\", \"size\": %d, \"seconds\": %.6f, \"level_rows\": [",
                 vfb_status_str(res.status), res.size, res.seconds);
    for (int k = 1; k <= res.size; ++k)
      std::fprintf(stderr, "%s%llu", k > 1 ? ", " : "", (unsigned long long)res.level_rows[k]);
    std::fprintf(stderr, "], \"level_cands\": [");
    for (int k = 1; k <= res.size; ++k)
      std::fprintf(stderr, "%s%llu", k > 1 ? ", " : "", (unsigned long long)res.level_cands[k]);
    std::fprintf(stderr, "]}\n");
  }
  vfb_destroy(ctx);
  vfb_json_free(jp);
  return rc;
}
