// main.cpp - the es_b200 command: the reference's executable interface
// (src/main.cpp:31-93) on the CUDA backend.
//
//   es_b200                -- run default.config
//   es_b200 <config_file>  -- run a config file
//   es_b200 help           -- usage
#include <cstdio>
#include <cstring>
#include <string>

#include "es_host.h"

int main(int argc, char** argv)
{
    std::string config = "default.config";
    if (argc >= 2) {
        if (std::strcmp(argv[1], "help") == 0) {
            std::printf("Usage:\n\n");
            std::printf("\tes_b200               -- Run a simulation with default.config as configuration.\n");
            std::printf("\tes_b200 [config_file] -- Use a custom config file.\n");
            std::printf("\tes_b200 help          -- Display usage.\n");
            return 0;
        }
        config = argv[1];
    }
    const es_status st = es_run_config(config.c_str(), nullptr, 0, 0);
    if (st != ES_OK) {
        std::fprintf(stderr, "%s\n", es_host_last_error());
        return 1;
    }
    return 0;
}
