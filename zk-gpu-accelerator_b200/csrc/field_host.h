// field_host.h — host-side field helpers shared by the .cu files.
#pragma once
#include "common.cuh"
#include "field.cuh"

namespace zkb {

int field_init(zkb_field* f, const uint64_t modulus[4]);
FieldRT to_rt(const zkb_field& f);
int check_field(const zkb_field* f);

// Calls fn with the field policy matching f: compile-time constants for
// BN254's two fields, runtime parameters for any other modulus.
template <class Fn>
int with_field(const zkb_field* f, Fn&& fn) {
  switch (f->kind) {
    case ZKB_FIELD_BN254_FR:
      return fn(FrP{});
    case ZKB_FIELD_BN254_FQ:
      return fn(FqP{});
    default:
      return fn(to_rt(*f));
  }
}

}  // namespace zkb
