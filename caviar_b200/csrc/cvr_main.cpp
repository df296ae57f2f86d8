// caviar_b200_casl: run a CASL script on the B200 path, like the reference's
// `CAVIAR -i script.casl` (src/main_CAVIAR.cpp:27-58) for the hot-path objects.
#include <cstdio>
#include <cstring>

#include "../../include/caviar_b200.h"

int main(int argc, char **argv) {
  const char *script = nullptr;
  for (int i = 1; i < argc; ++i)
    if (std::strcmp(argv[i], "-i") == 0 && i + 1 < argc) script = argv[++i];
  if (!script && argc == 2) script = argv[1];
  if (!script) {
    std::fprintf(stderr, "usage: %s -i script.casl\n", argv[0]);
    return 2;
  }
  char err[1024];
  const int rc = cvr_casl_run_file(script, err, sizeof(err));
  if (rc != CVR_OK) {
    std::fprintf(stderr, "[ERR] %s\n", err);
    return 1;
  }
  return 0;
}
