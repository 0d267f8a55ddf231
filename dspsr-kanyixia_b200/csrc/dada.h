// dada.h -- internal view of the DADA file source for the pipeline driver
#pragma once
#include "dspsr_b200.h"

namespace dspsr_b200_host
{
// records the message of a failed host-only call (dspsr_b200_host_error)
// and returns code
int host_fail (int code, const char* fmt, ...);

// the observation parameters loaded when the file was opened
const dspsr_b200_dada_info& dada_info (const dspsr_b200_dada_file* file);
}
