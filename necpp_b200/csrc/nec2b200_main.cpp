// nec2b200: the deck-file command line of libnecpp_b200 (the options of
// nec2++, src/nec2cpp.cpp:186-280): -i <input deck> [-o <output file>].
// Without -o the output goes to standard output.
#include <cstdio>
#include <cstring>
#include <string>

#include "include/libnecpp.h"

static void usage() {
  std::fprintf(stderr, "usage: nec2b200 -i <input.nec> [-o <output.out>]\n");
}

int main(int argc, char** argv) {
  std::string in, out;
  for (int k = 1; k < argc; k++) {
    if (!std::strcmp(argv[k], "-i") && k + 1 < argc) {
      in = argv[++k];
    } else if (!std::strcmp(argv[k], "-o") && k + 1 < argc) {
      out = argv[++k];
    } else if (!std::strcmp(argv[k], "-h")) {
      usage();
      return 0;
    } else {
      usage();
      return 2;
    }
  }
  if (in.empty()) {
    usage();
    return 2;
  }
  const long rc = nec_run_deck(in.c_str(), out.c_str());
  if (rc != 0) std::fprintf(stderr, "nec2b200: %s\n", nec_deck_error());
  return rc == 0 ? 0 : 1;
}
