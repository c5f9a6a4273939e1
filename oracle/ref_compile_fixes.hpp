// Compile fix shared by the test-only reference programs (ref_runner,
// ref_xml): DispersiveAtomicUpdate (include/DispersiveMaterials.hpp:260-282)
// puts enable_if on a class template parameter, which g++13 rejects when any
// material functor is instantiated. These partial specialisations forward to
// UpdateStruct::implicit_update / explicit_update with the same argument
// order as :272-280. The reference itself is not modified.
#pragma once
#include <fdtd.h>
#include <utility>

namespace fdtd {
template <typename U, typename F>
struct DispersiveAtomicUpdate<U, true, F> {
  static constexpr Dir d = FieldDir<F>::value;
  static constexpr FieldType ft = F::field_type;
  typedef typename FluxComponent<ft, d>::type DType;
  typedef typename FieldComponent<ft, d>::type EType;
  typedef typename CurrentComponent<ft, d>::type JType;
  typedef typename PolarizationComponent<ft, d>::type PType;
  template <typename T, typename... Args>
  static void get(T&& f, Args&&... args) {
    U::implicit_update(GetField<DType>::get(f), GetField<EType>::get(f),
                       GetField<PType>::get(f), GetField<JType>::get(f),
                       std::forward<Args>(args)...);
  }
};
template <typename U, typename F>
struct DispersiveAtomicUpdate<U, false, F> {
  static constexpr Dir d = FieldDir<F>::value;
  static constexpr FieldType ft = F::field_type;
  typedef typename FluxComponent<ft, d>::type DType;
  typedef typename FieldComponent<ft, d>::type EType;
  typedef typename CurrentComponent<ft, d>::type JType;
  typedef typename PolarizationComponent<ft, d>::type PType;
  template <typename T, typename... Args>
  static void get(T&& f, Args&&... args) {
    U::explicit_update(GetField<DType>::get(f), GetField<EType>::get(f),
                       GetField<PType>::get(f), GetField<JType>::get(f),
                       std::forward<Args>(args)...);
  }
};
}  // namespace fdtd
