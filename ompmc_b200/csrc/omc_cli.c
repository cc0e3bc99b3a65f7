/*
 * omc_dosxyz — drop-in for ompMC's CLI (omc_dosxyz.c:1072-1307):
 *
 *   omc_dosxyz -i <input without .inp> -o <output name> [--verbose|--brief]
 *              [--mode plain|event]
 *
 * Reads the same `.inp` keys and writes `<output folder><name>.3ddose`.
 * --mode selects the transport form (default: event, FP32 transport with
 * FP64 tallies; plain is FP64 history-based).  Exit status 0 on success, 1
 * on any error (the message goes to stderr).
 */
#include <getopt.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "omcgpu.h"

static int verbose_flag = 0;

int main(int argc, char **argv) {
    const char *input = NULL, *output = NULL;
    int mode = OMC_EVENT_FP32;
    static struct option opts[] = {
        {"verbose", no_argument, &verbose_flag, 1},
        {"brief", no_argument, &verbose_flag, 0},
        {"input", required_argument, 0, 'i'},
        {"output", required_argument, 0, 'o'},
        {"mode", required_argument, 0, 'm'},
        {0, 0, 0, 0},
    };
    for (;;) {
        int idx = 0;
        int c = getopt_long(argc, argv, "i:o:m:", opts, &idx);
        if (c == -1) break;
        switch (c) {
            case 0: break;
            case 'i': input = optarg; break;
            case 'o': output = optarg; break;
            case 'm':
                if (!strcmp(optarg, "plain")) mode = OMC_PLAIN_FP64;
                else if (!strcmp(optarg, "event")) mode = OMC_EVENT_FP32;
                else {
                    fprintf(stderr, "unknown --mode %s (plain|event)\n", optarg);
                    return 1;
                }
                break;
            default: return 1;
        }
    }
    if (!input || !output) {
        fprintf(stderr, "usage: %s -i <input> -o <output> [--verbose] [--mode plain|event]\n", argv[0]);
        return 1;
    }
    int rc = omc_dosxyz_run(input, output, mode, verbose_flag);
    if (rc != OMC_OK) {
        fprintf(stderr, "omc_dosxyz failed: %s (%d)\n", omc_status_string(rc), rc);
        return 1;
    }
    return 0;
}
