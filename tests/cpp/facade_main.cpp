// Drives a registration through the reg:: C++ facade (include/claire_b200.hpp)
// for tests/test_facade.py.
//   facade_main opts <args...>            print the parsed options
//   facade_main run <dir> <args...>       read <dir>/mR.bin, mT.bin (nl floats),
//                                         register, write <dir>/v.bin and the
//                                         preconditioner applied to v, <dir>/pv.bin,
//                                         and print stats
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "claire_b200.hpp"

static bool read_file(const std::string& p, std::vector<float>& out) {
  FILE* f = std::fopen(p.c_str(), "rb");
  if (!f) return false;
  const size_t got = std::fread(out.data(), sizeof(float), out.size(), f);
  std::fclose(f);
  return got == out.size();
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string mode = argv[1];
  if (mode == "opts") {
    std::vector<char*> args = {argv[0]};
    for (int i = 2; i < argc; ++i) args.push_back(argv[i]);
    reg::RegOpt opt((int)args.size(), args.data());
    const claire_b200_opts& o = opt.opts();
    std::printf("{\"status\": %d, \"nx\": [%d, %d, %d], \"nt\": %d, \"regnorm\": %d, \"beta\": %.17g, "
                "\"maxit\": %d, \"opttol\": %.17g, \"distance\": %d, \"bytes\": %lld}\n",
                opt.status(), o.nx[0], o.nx[1], o.nx[2], o.nt, o.regnorm, o.beta[0], o.maxit, o.opttol, o.distance,
                opt.EstimateBytes(1));
    return opt.status() == 0 ? 0 : 1;
  }
  if (mode == "run" && argc >= 3) {
    const std::string dir = argv[2];
    std::vector<char*> args = {argv[0]};
    for (int i = 3; i < argc; ++i) args.push_back(argv[i]);
    reg::RegOpt opt((int)args.size(), args.data());
    if (opt.status()) return 3;
    std::vector<float> mR(opt.nl()), mT(opt.nl());
    if (!read_file(dir + "/mR.bin", mR) || !read_file(dir + "/mT.bin", mT)) return 4;
    reg::CLAIREInterface reg(&opt);
    if (reg.status()) {
      std::fprintf(stderr, "create: %d\n", reg.status());
      return 5;
    }
    if (reg.SetReferenceImage(mR.data()) || reg.SetTemplateImage(mT.data())) return 6;
    if (int e = reg.Run()) {
      std::fprintf(stderr, "run: %d %s\n", e, reg.LastError());
      return 7;
    }
    reg::VecField v(opt);
    if (reg.GetSolution(&v)) return 8;
    reg::Preconditioner pc(&reg);
    reg::VecField pv(opt);
    if (pc.MatVec(&pv, &v)) return 11;
    FILE* fp = std::fopen((dir + "/pv.bin").c_str(), "wb");
    if (!fp) return 10;
    std::fwrite(pv.data(), sizeof(float), 3 * pv.nl(), fp);
    std::fclose(fp);
    double det[3];
    if (reg.ComputeDetDefGrad(nullptr, det)) return 9;
    claire_b200_stats st;
    reg.GetStats(&st);
    FILE* f = std::fopen((dir + "/v.bin").c_str(), "wb");
    if (!f) return 10;
    std::fwrite(v.data(), sizeof(float), 3 * v.nl(), f);
    std::fclose(f);
    std::printf("{\"gn\": %d, \"pcg\": %d, \"mismatch\": %.17g, \"det_min\": %.9g, \"det_max\": %.9g}\n",
                st.gn_iterations, st.pcg_iterations, st.rel_mismatch, det[0], det[2]);
    return 0;
  }
  return 2;
}
