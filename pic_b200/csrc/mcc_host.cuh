// Host-side owner of the MCC device tables (shared by mcc.cu and step.cu).
#pragma once

#include <vector>

#include "mcc.cuh"

namespace pic {

struct MccHost {
    MccDev dev{};
    double nu_max[PIC_MAX_SPECIES] = {};
    double p_null[PIC_MAX_SPECIES] = {};
    std::vector<void*> allocs;
};

// Uploads the tables and computes nu' and P_null per species (species masses in kg).
int mcc_build(const pic_mcc_desc* d, int nspecies, const double* mass, double dt, MccHost* H);
void mcc_free(MccHost* H);

}  // namespace pic
