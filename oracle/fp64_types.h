/*
 * Pre-included (-include) when building the FP64 oracles. It claims the
 * reference's PrecisionTypes.h include guard and makes every FP type double,
 * which is the switch the reference's include/PrecisionTypes.h:4-10 offers.
 * TEST INFRASTRUCTURE ONLY.
 */
#ifndef PRECISIONTYPES_H
#define PRECISIONTYPES_H
typedef double FPpart;
typedef double FPfield;
typedef double FPinterp;
#endif
