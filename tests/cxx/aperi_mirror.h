// aperi_mirror.h -- the reference's element / force-contribution interface, restated
// with the same class names and virtual signatures so that the shim aperi-mech would
// compile (b200_element.h) compiles here against include/aperi_b200.h.
//
//   aperi::ElementBase::ComputeInternalForceAllElements(double time_increment, double time)
//       include/ElementBase.h:75 (pure virtual)
//   aperi::ForceContribution::ComputeForce(Field<Real>&, double time, double time_increment)
//       include/ForceContribution.h:28 (pure virtual)
//   aperi::InternalForceContribution::ComputeForce -> m_element->ComputeInternalForceAllElements
//       include/InternalForceContribution.h:49-53
//
// In the reference the fields live in STK and the element finds them by name; here a
// Field is a caller-owned device array of N x 3 doubles (a 3-component node field,
// include/Field.h:129-136), handed to the element when it is created.
#pragma once

#include <cstddef>
#include <memory>
#include <stdexcept>
#include <utility>

namespace aperi {

using Real = double;

template <typename T>
class Field {
   public:
    Field(T* device_data, size_t num_nodes) : m_data(device_data), m_num_nodes(num_nodes) {}
    T* data() { return m_data; }
    const T* data() const { return m_data; }
    size_t NumNodes() const { return m_num_nodes; }

   private:
    T* m_data;
    size_t m_num_nodes;
};

class ElementBase {
   public:
    explicit ElementBase(size_t num_nodes) : m_num_nodes(num_nodes) {}
    virtual ~ElementBase() = default;
    size_t GetNumNodes() const { return m_num_nodes; }
    virtual void ComputeInternalForceAllElements(double time_increment, double time) = 0;
    virtual void PopulateElementOutputs() {}

   protected:
    size_t m_num_nodes;
};

class ForceContribution {
   public:
    ForceContribution() = default;
    virtual ~ForceContribution() = default;
    virtual void Preprocess() {}
    virtual void ComputeForce(Field<Real>& force_field, double time, double time_increment) = 0;
};

class InternalForceContribution : public ForceContribution {
   public:
    explicit InternalForceContribution(std::shared_ptr<ElementBase> element) : m_element(std::move(element)) {
        if (!m_element) throw std::invalid_argument("InternalForceContribution needs an element");
    }
    void ComputeForce(Field<Real>& /*force_field*/, double time, double time_increment) override {
        m_element->ComputeInternalForceAllElements(time_increment, time);
    }
    std::shared_ptr<ElementBase> GetElement() const { return m_element; }

   private:
    std::shared_ptr<ElementBase> m_element;
};

}  // namespace aperi
