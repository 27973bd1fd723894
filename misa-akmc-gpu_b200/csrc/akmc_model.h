// akmc_model.h -- host-side model construction (internal).
#pragma once

#include <stdint.h>

#include <vector>

#include "akmc_device.h"

namespace akmc {

int shells_within(double lattice_const, double cutoff);
void build_geometry(Geometry& g, int nshells);
void pairbond_tables(double b1[5][5], double b2[5][5]);
void cell_coefs(const double* F, int n, int k, double c[4]);
int eam_johnson(uint64_t seed, double lattice_const, double cutoff, akmc_eam_tables* out, double params[4][5]);
// Fills P (tables, no device pointers), the FP64 F coefficients and the FP32 cells.
int build_potential(const akmc_eam_tables* t, Potential& P, std::vector<double>& coef, std::vector<FCell32>& f32);
// Reference rank split of n cells over p blocks: start[k] = k (n/p) + min(k, n % p).
void block_split(int64_t n, int p, std::vector<int32_t>& start);
int create_lattice(const int64_t box[3], const int32_t codes[4], const int64_t ratio[4], int64_t nvac, uint64_t seed,
                   uint8_t* occ, int64_t n);
int cluster_stats(const uint8_t* occ, const int64_t box[3], int64_t* isolated, int64_t* hist, int64_t hist_len);

}  // namespace akmc
