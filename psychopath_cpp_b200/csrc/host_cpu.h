/*
 * Host-CPU dependent constants (see host_cpu.cpp).
 */
#ifndef PSY_HOST_CPU_H
#define PSY_HOST_CPU_H

namespace psy {

// Diagonal of the reference's inverse of the identity matrix on this CPU.
float reference_identity_inverse_scale();

}  // namespace psy

#endif
