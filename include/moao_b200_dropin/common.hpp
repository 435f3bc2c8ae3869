/*
 * Drop-in for the reference's common/common.hpp (common/common.hpp:1-20).
 *
 * Put this directory first on the include path of the reference's own drivers
 * (lapack/moao_lapack.cpp, lapack/check_moao_lapack.cpp) and link them against
 * libmoao_b200.so instead of the reference's common library: Tomo_struct,
 * MOAO_COMMON::matcov_tile, MOAO_LAPACK::reconstructor / Cee_Cvv / geadd, the
 * intersample entry points and the FITS helpers then come from this library
 * (moao_b200_compat.hpp), while the drivers keep the reference's own
 * command-line, timer and matrix-comparison utilities (common/io/arguments.hpp,
 * common/utils/timer.hpp, common/compute/check_utils.hpp, compiled from the
 * reference tree with the driver).
 * The standard headers are those the reference's common headers bring in.
 */
#ifndef COMMON_H
#define COMMON_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "moao_b200_compat.hpp"
#include "compute/check_utils.hpp"
#include "io/arguments.hpp"
#include "utils/timer.hpp"

#endif  // COMMON_H
