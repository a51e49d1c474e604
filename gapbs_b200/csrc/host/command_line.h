// command_line.h -- the pr_spmv command-line surface for the pr_gpu CLI and
// the graph C ABI.
//
// Accepts the same options, with the same defaults, help text and bundling
// rules as the reference's CLBase -> CLApp -> CLPageRank chain
// (src/command_line.h:28-197; option string "f:g:hk:su:m" + "an:r:vl" +
// "i:t:"): -f file, -g/-u scale, -k degree, -s, -m, -a, -n trials, -r node,
// -v, -l, -i max iterations, -t tolerance, -h.  "-g10 -vn1" style bundles
// parse as getopt parses them.  Unknown letters are reported and skipped,
// as getopt does.  Built with iterative = false it is the reference's plain
// CLApp (no -i / -t), the command line of its cc binary.
#ifndef GAPBS_B200_HOST_COMMAND_LINE_H_
#define GAPBS_B200_HOST_COMMAND_LINE_H_

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "builder.h"

namespace gapbs_b200 {

class PageRankCLI {
 public:
  PageRankCLI(std::string name, double tolerance, int max_iters, bool iterative = true)
      : name_(name), tolerance_(tolerance), max_iters_(max_iters), iterative_(iterative) {
    Help('h', "", "print this help message");
    Help('f', "file", "load graph from file");
    Help('s', "", "symmetrize input edge list", "false");
    Help('g', "scale", "generate 2^scale kronecker graph");
    Help('u', "scale", "generate 2^scale uniform-random graph");
    Help('k', "degree", "average degree for synthetic graph", std::to_string(src_.degree));
    Help('m', "", "reduces memory usage during graph building", "false");
    Help('a', "", "output analysis of last run", "false");
    Help('n', "n", "perform n trials", std::to_string(num_trials_));
    Help('r', "node", "start from node r", "rand");
    Help('v', "", "verify the output of each run", "false");
    Help('l', "", "log performance within each trial", "false");
    if (iterative_) {
      Help('i', "i", "perform at most i iterations", std::to_string(max_iters_));
      Help('t', "t", "use tolerance t", std::to_string(tolerance_));
    }
  }

  // Returns false (after printing the reference's message) when no graph
  // input was given.  -h prints usage and exits 0, as the reference does.
  bool Parse(int argc, char **argv) {
    const std::string with_arg = iterative_ ? "fgkunrit" : "fgkunr";
    const std::string flags = "hsmavl";
    for (int i = 1; i < argc; i++) {
      const char *tok = argv[i];
      if (tok[0] != '-' || tok[1] == '\0') continue;
      for (int j = 1; tok[j] != '\0'; j++) {
        char c = tok[j];
        if (with_arg.find(c) != std::string::npos) {
          std::string arg;
          if (tok[j + 1] != '\0') {
            arg = tok + j + 1;
          } else if (i + 1 < argc) {
            arg = argv[++i];
          } else {
            std::fprintf(stderr, "%s: option requires an argument -- '%c'\n", argv[0], c);
            break;
          }
          Handle(c, arg);
          break;
        } else if (flags.find(c) != std::string::npos) {
          Handle(c, "");
        } else {
          std::fprintf(stderr, "%s: invalid option -- '%c'\n", argv[0], c);
        }
      }
    }
    if (src_.filename.empty() && src_.scale == -1) {
      std::cout << "No graph input specified. (Use -h for help)" << std::endl;
      return false;
    }
    if (src_.scale != -1) src_.symmetrize = true;
    return true;
  }

  const GraphSource &source() const { return src_; }
  bool do_analysis() const { return do_analysis_; }
  int num_trials() const { return num_trials_; }
  int64_t start_vertex() const { return start_vertex_; }
  bool do_verify() const { return do_verify_; }
  bool logging_en() const { return logging_; }
  int max_iters() const { return max_iters_; }
  double tolerance() const { return tolerance_; }

 private:
  void Handle(char c, const std::string &arg) {
    switch (c) {
      case 'f': src_.filename = arg; break;
      case 'g': src_.scale = std::atoi(arg.c_str()); break;
      case 'h': PrintUsage(); break;
      case 'k': src_.degree = std::atoi(arg.c_str()); break;
      case 's': src_.symmetrize = true; break;
      case 'u': src_.uniform = true; src_.scale = std::atoi(arg.c_str()); break;
      case 'm': src_.in_place = true; break;
      case 'a': do_analysis_ = true; break;
      case 'n': num_trials_ = std::atoi(arg.c_str()); break;
      case 'r': start_vertex_ = std::atol(arg.c_str()); break;
      case 'v': do_verify_ = true; break;
      case 'l': logging_ = true; break;
      case 'i': max_iters_ = std::atoi(arg.c_str()); break;
      case 't': tolerance_ = std::stod(arg); break;
    }
  }

  void Help(char opt, std::string opt_arg, std::string text, std::string def = "") {
    char buf[100];
    if (!opt_arg.empty()) opt_arg = "<" + opt_arg + ">";
    if (!def.empty()) def = "[" + def + "]";
    std::snprintf(buf, sizeof(buf), " -%c %-9s: %-54s%10s", opt, opt_arg.c_str(),
                  text.c_str(), def.c_str());
    help_.push_back(buf);
  }

  void PrintUsage() {
    std::cout << name_ << std::endl;
    for (const std::string &h : help_) std::cout << h << std::endl;
    std::exit(0);
  }

  std::string name_;
  GraphSource src_;
  bool do_analysis_ = false;
  int num_trials_ = 16;
  int64_t start_vertex_ = -1;
  bool do_verify_ = false;
  bool logging_ = false;
  double tolerance_;
  int max_iters_;
  bool iterative_;
  std::vector<std::string> help_;
};

}  // namespace gapbs_b200

#endif  // GAPBS_B200_HOST_COMMAND_LINE_H_
