// grb_semirings.h: the built-in semirings compiled for the device, one line
// each, as (add monoid opcode, multiply opcode, type code, C++ type).  The
// list is closed under the operand swap the drop-in boundary performs
// (FIRST <-> SECOND, FIRSTI <-> SECONDJ, FIRSTJ <-> SECONDI).  It mirrors the
// factory kernels the reference ships for the configs of
// this path (FactoryKernels/GB_AxB__plus_times_fp64.c, __plus_pair_int64.c,
// __min_plus_fp32.c, __any_firstj_int64.c) plus the common variants of each;
// any other semiring is declined with GrB_NO_VALUE so the caller can take
// its own path, as the reference's GPU gateway declines what it cannot run.

#pragma once

#define GRB_FOR_EACH_SEMIRING(X)                     \
    X(OP_PLUS,  OP_TIMES,   T_FP64,  double)         \
    X(OP_PLUS,  OP_TIMES,   T_FP32,  float)          \
    X(OP_PLUS,  OP_TIMES,   T_INT64, int64_t)        \
    X(OP_PLUS,  OP_TIMES,   T_INT32, int32_t)        \
    X(OP_PLUS,  OP_PAIR,    T_INT64, int64_t)        \
    X(OP_PLUS,  OP_PAIR,    T_INT32, int32_t)        \
    X(OP_PLUS,  OP_PAIR,    T_FP64,  double)         \
    X(OP_MIN,   OP_PLUS,    T_FP32,  float)          \
    X(OP_MIN,   OP_PLUS,    T_FP64,  double)         \
    X(OP_MIN,   OP_PLUS,    T_INT64, int64_t)        \
    X(OP_MIN,   OP_PLUS,    T_INT32, int32_t)        \
    X(OP_MAX,   OP_PLUS,    T_FP64,  double)         \
    X(OP_MAX,   OP_PLUS,    T_FP32,  float)          \
    X(OP_MIN,   OP_TIMES,   T_FP64,  double)         \
    X(OP_MAX,   OP_TIMES,   T_FP64,  double)         \
    X(OP_MIN,   OP_SECOND,  T_FP32,  float)          \
    X(OP_MIN,   OP_SECOND,  T_FP64,  double)         \
    X(OP_MIN,   OP_FIRST,   T_FP32,  float)          \
    X(OP_MIN,   OP_FIRST,   T_FP64,  double)         \
    X(OP_PLUS,  OP_FIRST,   T_FP64,  double)         \
    X(OP_PLUS,  OP_SECOND,  T_FP64,  double)         \
    X(OP_ANY,   OP_SECONDI, T_INT64, int64_t)        \
    X(OP_ANY,   OP_FIRSTJ,  T_INT64, int64_t)        \
    X(OP_ANY,   OP_FIRSTI,  T_INT64, int64_t)        \
    X(OP_ANY,   OP_SECONDJ, T_INT64, int64_t)        \
    X(OP_ANY,   OP_SECONDI, T_INT32, int32_t)        \
    X(OP_ANY,   OP_FIRSTJ,  T_INT32, int32_t)        \
    X(OP_MIN,   OP_SECONDI, T_INT64, int64_t)        \
    X(OP_MIN,   OP_FIRSTJ,  T_INT64, int64_t)        \
    X(OP_MIN,   OP_FIRSTI,  T_INT64, int64_t)        \
    X(OP_MIN,   OP_SECONDJ, T_INT64, int64_t)        \
    X(OP_MAX,   OP_SECONDI, T_INT64, int64_t)        \
    X(OP_MAX,   OP_FIRSTJ,  T_INT64, int64_t)        \
    X(OP_ANY,   OP_PAIR,    T_BOOL,  bool)           \
    X(OP_LOR,   OP_LAND,    T_BOOL,  bool)           \
    X(OP_ANY,   OP_PAIR,    T_INT64, int64_t)        \
    X(OP_ANY,   OP_TIMES,   T_FP64,  double)
