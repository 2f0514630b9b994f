/*
 * Tables of the Faure-permuted Halton sequence (see sampler_tables.cpp).
 */
#ifndef PSY_SAMPLER_TABLES_H
#define PSY_SAMPLER_TABLES_H

#include <cstdint>
#include <vector>

#define PSY_HALTON_DIMS 256

namespace psy {

struct HaltonDim {
	uint32_t base;
	uint32_t pow_base;     // base^digits (<= 500)
	uint32_t groups;       // digit groups covering 32 bits
	uint32_t perm_offset;  // first entry in the permutation pool
};

struct HaltonTables {
	std::vector<HaltonDim> dims;   // PSY_HALTON_DIMS
	std::vector<double> cmul;      // (1 - 2^-24) / max_power per dimension
	std::vector<uint16_t> perm;    // concatenated permutation tables
};

HaltonTables build_halton_tables();

}  // namespace psy

#endif
