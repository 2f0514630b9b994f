/*
 * Host-CPU dependent constants (see host_cpu.cpp).
 */
#ifndef PSY_HOST_CPU_H
#define PSY_HOST_CPU_H

#include <cstdint>
#include <vector>

#include "psy_math.h"

namespace psy {

// Diagonal of the reference's inverse of the identity matrix on this CPU.
float reference_identity_inverse_scale();

// This CPU's approximate reciprocal instruction as a table (psy_math.h
// RcpTable), built and checked once per process.  `entries` is the table's
// host copy, which the contexts upload to their devices.
struct HostRcp {
	std::vector<uint32_t> entries;
	int shift;
	RcpTable table() const { return RcpTable{entries.data(), shift}; }
};
const HostRcp& host_rcp();

}  // namespace psy

#endif
