// poststackmig <config.txt> -- the reference's command line (src/main.cpp:66-70, 438-441)
// with the migration on the GPU.  Exit 0 on success, 1 with "Error: ..." on stderr.
#include <cstdio>
#include <iostream>

#include "psm_host.h"

int main(int argc, char** argv) {
    if (argc != 2) {
        std::cerr << "Usage: " << argv[0] << " <config_file>" << std::endl;
        return 1;
    }
    char err[2048];
    if (psm_run_config(argv[1], 1, err, sizeof err) != 0) {
        std::cerr << "Error: " << err << std::endl;
        return 1;
    }
    return 0;
}
