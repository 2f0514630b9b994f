/*
 * Halton sequence with Faure digit permutations (L. Gruenschloss'
 * construction, the one behind the reference's generated
 * sampling/halton.cpp: 256 dimensions, one prime base per dimension,
 * radical inverse evaluated a few digits at a time through permutation
 * tables of at most 500 entries).
 *
 * Per dimension with prime base b:
 *   digits   = largest k with b^k <= 500, pow_base = b^k;
 *   max_power = the largest power of pow_base below 2^32;
 *   perm[j]  = Faure-permuted radical inverse of j over `digits` digits;
 *   sample(i) = float( double(sum_g perm[(i / pow_base^g) % pow_base] *
 *                              max_power / pow_base^(g+1))
 *                      * ((1 - 2^-24) / max_power) ).
 * Base 2 is the bit reversal of the index scaled by 2^-32.
 *
 * Faure permutations: sigma_2 = (0 1); for odd b, sigma_b inserts the
 * centre c = (b-1)/2 into sigma_{b-1} shifted around c; for even b = 2c,
 * sigma_b(i) = 2 sigma_c(i) for i < c and 2 sigma_c(i-c) + 1 otherwise.
 */
#include "sampler_tables.h"

#include <cstdint>
#include <vector>

namespace psy {

namespace {

std::vector<uint32_t> first_primes(int count) {
	std::vector<uint32_t> p;
	for (uint32_t c = 2; (int)p.size() < count; ++c) {
		bool prime = true;
		for (uint32_t d = 2; d * d <= c; ++d)
			if (c % d == 0) {
				prime = false;
				break;
			}
		if (prime) p.push_back(c);
	}
	return p;
}

}  // namespace

HaltonTables build_halton_tables() {
	HaltonTables t;
	const std::vector<uint32_t> primes = first_primes(PSY_HALTON_DIMS);
	const uint32_t maxb = primes.back();
	// Faure permutations for every base up to the largest prime.
	std::vector<std::vector<uint32_t>> faure(maxb + 1);
	faure[0] = {0};
	faure[1] = {0};
	faure[2] = {0, 1};
	for (uint32_t b = 3; b <= maxb; ++b) {
		std::vector<uint32_t>& f = faure[b];
		f.resize(b);
		if (b & 1) {
			const uint32_t c = (b - 1) / 2;
			for (uint32_t i = 0; i < b; ++i) {
				if (i == c) {
					f[i] = c;
				} else {
					const uint32_t v = faure[b - 1][i - (i > c ? 1 : 0)];
					f[i] = v + (v >= c ? 1 : 0);
				}
			}
		} else {
			const uint32_t c = b / 2;
			for (uint32_t i = 0; i < b; ++i) f[i] = i < c ? 2 * faure[c][i] : 2 * faure[c][i - c] + 1;
		}
	}
	for (int dim = 0; dim < PSY_HALTON_DIMS; ++dim) {
		const uint32_t base = primes[dim];
		HaltonDim hd{};
		hd.base = base;
		if (dim == 0) {
			t.dims.push_back(hd);
			t.cmul.push_back(0.0);
			continue;
		}
		uint32_t digits = 1;
		uint64_t pow_base = base;
		while (pow_base * base <= 500) {
			pow_base *= base;
			++digits;
		}
		uint64_t max_power = pow_base;
		int groups = 1;
		while (max_power * pow_base < (1ull << 32)) {
			max_power *= pow_base;
			++groups;
		}
		hd.pow_base = (uint32_t)pow_base;
		hd.groups = groups;
		hd.perm_offset = (uint32_t)t.perm.size();
		for (uint64_t j = 0; j < pow_base; ++j) {
			uint64_t idx = j, r = 0;
			for (uint32_t k = 0; k < digits; ++k) {
				const uint64_t rem = idx % base;
				idx /= base;
				r = r * base + faure[base][rem];
			}
			t.perm.push_back((uint16_t)r);
		}
		t.dims.push_back(hd);
		t.cmul.push_back(0x1.fffffep-1 / (double)max_power);
	}
	return t;
}

}  // namespace psy
