// spiffe_b200/csrc/spiffe_main.cpp -- the spiffe command line on the GPU:
//
//     spiffe-b200 [-threads=N] [-precision=f64|split32] inputfile
//
// as spiffe.c:92-365: the input file's commands run in order; the rootname
// is the input file's name up to its first '.'.  -threads is accepted for
// compatibility (the reference's OpenMP thread count) and has no effect.
// Exit status 0, or 1 after &stop or an error.
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/spiffe_b200_session.h"

int main(int argc, char **argv)
{
  int precision = SPIFFE_PRECISION_F64;
  const char *input = nullptr;
  for (int i = 1; i < argc; i++) {
    if (std::strncmp(argv[i], "-threads=", 9) == 0)
      continue;
    if (std::strcmp(argv[i], "-precision=split32") == 0)
      precision = SPIFFE_PRECISION_SPLIT32;
    else if (std::strcmp(argv[i], "-precision=f64") == 0)
      precision = SPIFFE_PRECISION_F64;
    else if (!input && argv[i][0] != '-')
      input = argv[i];
    else {
      std::fprintf(stderr, "unknown argument %s\n", argv[i]);
      input = nullptr;
      break;
    }
  }
  if (!input) {
    std::fprintf(stderr, "usage: spiffe-b200 [-threads=N] [-precision=f64|split32] inputfile\n");
    return 1;
  }
  std::string root = input;
  const size_t dot = root.find('.');
  if (dot != std::string::npos)
    root.resize(dot);
  std::printf("Running spiffe_b200 (%s)\n", spiffe_gpu_version());
  spiffe_session *s = nullptr;
  if (spiffe_session_create(precision, root.c_str(), &s) != 0) {
    std::fprintf(stderr, "error: %s\n", spiffe_gpu_last_error());
    return 1;
  }
  const int rc = spiffe_session_run_file(s, input);
  if (rc < 0)
    std::fprintf(stderr, "error: %s\n", spiffe_gpu_last_error());
  const int rd = spiffe_session_destroy(s);
  if (rd < 0 && rc >= 0)
    std::fprintf(stderr, "error: %s\n", spiffe_gpu_last_error());
  return rc == 0 && rd == 0 ? 0 : 1;
}
