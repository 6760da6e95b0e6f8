// Library identity and status strings of the C ABI (include/rspi.h).
#include "rspi_common.cuh"

extern "C" const char *rspi_version(void) { return "rspi 0.1 sm_100a"; }

extern "C" const char *rspi_status_string(int status) {
    switch (status) {
        case RSPI_OK:
            return "ok";
        case RSPI_ERR_ARG:
            return "bad argument";
        case RSPI_ERR_INDEX:
            return "index out of range in the input";
        case RSPI_ERR_CUDA:
            return "CUDA launch failed";
        case RSPI_ERR_TIMEOUT:
            return "device-side wait timed out";
        case RSPI_ERR_CAPACITY:
            return "value does not fit the packed layout";
        case RSPI_ERR_TOO_LARGE:
            return "size exceeds the fixed scratch of a no-allocation entry point";
        default:
            return "unknown status";
    }
}
