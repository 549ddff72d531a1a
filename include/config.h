// config.h -- compile-time limb-width configuration of the multiply API,
// compatible with nikitaborisov/birdwing include/config.h:9-67.
//
// Three configurations are chosen with macros, as in the reference:
//   -DLIMB_BITS=32                       u32 limbs, 32-bit residues, 3 primes
//   -DLIMB_BITS=64                       u32 limbs, 64-bit residues, 2 primes
//   -DLIMB_BITS=64 -DNATIVE_HOST_LIMBS   u64 limbs, 64-bit residues, 3 primes
// They only select types for source compatibility: libbirdwing itself
// carries both prime paths and picks one at run time.
#pragma once
#ifndef CONFIG_H
#define CONFIG_H

#include <cstdint>
#include <type_traits>
#include <vector>

#ifndef LIMB_BITS
#define LIMB_BITS 32
#endif

#ifndef DEBUG
#define DEBUG 0
#endif

#if LIMB_BITS == 64 && defined(NATIVE_HOST_LIMBS)
#define NUM_MODULI 3
#define INPUT_LIMB_BITS 64
#define OUTPUT_LIMB_BITS 64
#define CRT_COEFF_BITS 160
#elif LIMB_BITS == 64
#define NUM_MODULI 2
#define INPUT_LIMB_BITS 32
#define OUTPUT_LIMB_BITS 32
#define CRT_COEFF_BITS 128
#else
#define NUM_MODULI 3
#define INPUT_LIMB_BITS 32
#define OUTPUT_LIMB_BITS 32
#define CRT_COEFF_BITS 128
#endif

#if LIMB_BITS == 64
using LimbType = uint64_t;
using TestDataTypeUint = uint64_t;
using TestDataTypeInt = int64_t;
#define LIMB_MASK 0xFFFFFFFFFFFFFFFFULL
#else
using LimbType = uint32_t;
using TestDataTypeUint = uint32_t;
using TestDataTypeInt = int32_t;
#define LIMB_MASK 0xFFFFFFFFULL
#endif

constexpr int BIT_WIDTH = sizeof(TestDataTypeUint) * 8;

using InputLimbType = std::conditional_t<INPUT_LIMB_BITS == 64, uint64_t, uint32_t>;
using OutputLimbType = std::conditional_t<OUTPUT_LIMB_BITS == 64, uint64_t, uint32_t>;

#if OUTPUT_LIMB_BITS == 64
#define OUTPUT_LIMB_MASK 0xFFFFFFFFFFFFFFFFULL
#else
#define OUTPUT_LIMB_MASK 0xFFFFFFFFULL
#endif

using namespace std;

#define BATCH 1
#define CARRY_SEG 1024

// RNS moduli and maximal-order roots of the configured width (defined by the
// compat library, or by a test that mirrors its own tables).
extern vector<TestDataTypeUint> moduli;
extern vector<TestDataTypeUint> roots_of_unity_max;

#endif  // CONFIG_H
