// b200_element.h -- the element shim a maintainer adds to aperi-mech: one part's
// ElementBase whose internal force is computed by libaperi_b200.so. It is the class
// INTEGRATION.md shows, compiled against the interface mirror (aperi_mirror.h) and the
// C ABI (include/aperi_b200.h).
#pragma once

#include <stdexcept>
#include <string>

#include "aperi_b200.h"
#include "aperi_mirror.h"

class B200Element : public aperi::ElementBase {
   public:
    // desc: the part's connectivity (reference node order, ShapeFunctionsFunctorHex8.h:17-33)
    // and completed Lame parameters (LinearElasticProperties, Materials/Base.h:47-129).
    // u: displacement_coefficients (state NP1), f: force_coefficients; N x 3 device arrays.
    B200Element(am_ctx* ctx, const am_block_desc& desc, size_t num_nodes, const aperi::Field<aperi::Real>& u,
                aperi::Field<aperi::Real>& f, am_precision precision = AM_FP64)
        : aperi::ElementBase(num_nodes), m_ctx(ctx), m_u(u.data()), m_f(f.data()), m_precision(precision) {
        if (am_add_block(ctx, &desc, &m_block) != AM_OK) throw std::runtime_error(am_last_error(ctx));
    }
    // The solver zeroes the force field and every contribution accumulates into it
    // (src/Solvers/Explicit.cpp:157-163): accumulate = 1 keeps that contract.
    void ComputeInternalForceAllElements(double /*time_increment*/, double /*time*/) override {
        const int rc = am_internal_force(m_ctx, m_precision, AM_DEVICE, m_u, m_f, /*accumulate=*/1);
        if (rc != AM_OK) throw std::runtime_error(std::string("am_internal_force: ") + am_last_error(m_ctx));
    }
    int32_t Block() const { return m_block; }

   private:
    am_ctx* m_ctx;
    const double* m_u;
    double* m_f;
    am_precision m_precision;
    int32_t m_block = -1;
};
