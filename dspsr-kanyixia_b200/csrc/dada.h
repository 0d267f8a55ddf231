// dada.h -- internal view of the DADA file source for the pipeline driver
#pragma once
#include "dspsr_b200.h"

namespace dspsr_b200_host
{
// the observation parameters loaded when the file was opened
const dspsr_b200_dada_info& dada_info (const dspsr_b200_dada_file* file);
}
