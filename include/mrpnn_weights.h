/*
 * mrpnn_weights.h - flat weight blob layout of the radiance-predictor MLP.
 *
 * The blob is 49,673 fp32 values: the named arrays of the reference's weight
 * header (core/NNWeight.cuh:1-439) concatenated in their declaration order.
 * Matrices are stored [out][in] row-major (element (i, j) of a From->To layer
 * is W[j + i*From], core/radiancePredict.cu:51), biases separately.
 * The order and sizes below must stay identical to that header so that a
 * weight file written for the reference loads unchanged.
 */
#ifndef MRPNN_WEIGHTS_H
#define MRPNN_WEIGHTS_H

#define MR_WEIGHT_LIST(X) \
  X(LD01W, 64) \
  X(LD01B, 8) \
  X(LD11W, 64) \
  X(LD11B, 8) \
  X(LD21W, 64) \
  X(LD21B, 8) \
  X(LD31W, 64) \
  X(LD31B, 8) \
  X(LD41W, 64) \
  X(LD41B, 8) \
  X(LD_Tr01W, 64) \
  X(LD_Tr01B, 8) \
  X(LD_Tr11W, 64) \
  X(LD_Tr11B, 8) \
  X(LD_Tr21W, 64) \
  X(LD_Tr21B, 8) \
  X(LD_Tr31W, 64) \
  X(LD_Tr31B, 8) \
  X(LD_Tr41W, 64) \
  X(LD_Tr41B, 8) \
  X(LD_Hg01W, 64) \
  X(LD_Hg01B, 8) \
  X(LD_Hg11W, 64) \
  X(LD_Hg11B, 8) \
  X(LD_Hg21W, 64) \
  X(LD_Hg21B, 8) \
  X(LD_Hg31W, 64) \
  X(LD_Hg31B, 8) \
  X(LD_Hg41W, 64) \
  X(LD_Hg41B, 8) \
  X(L01W, 64) \
  X(L01B, 8) \
  X(L11W, 64) \
  X(L11B, 8) \
  X(L21W, 256) \
  X(L21B, 16) \
  X(L31W, 256) \
  X(L31B, 16) \
  X(L41W, 256) \
  X(L41B, 16) \
  X(L51W, 1024) \
  X(L51B, 32) \
  X(L61W, 1024) \
  X(L61B, 32) \
  X(L71W, 1024) \
  X(L71B, 32) \
  X(L81W, 1024) \
  X(L81B, 32) \
  X(L_Tr01W, 64) \
  X(L_Tr01B, 8) \
  X(L_Tr11W, 64) \
  X(L_Tr11B, 8) \
  X(L_Tr21W, 256) \
  X(L_Tr21B, 16) \
  X(L_Tr31W, 256) \
  X(L_Tr31B, 16) \
  X(L_Tr41W, 256) \
  X(L_Tr41B, 16) \
  X(L_Tr51W, 1024) \
  X(L_Tr51B, 32) \
  X(L_Tr61W, 1024) \
  X(L_Tr61B, 32) \
  X(L_Tr71W, 1024) \
  X(L_Tr71B, 32) \
  X(L_Tr81W, 1024) \
  X(L_Tr81B, 32) \
  X(L_Hg01W, 64) \
  X(L_Hg01B, 8) \
  X(L_Hg11W, 64) \
  X(L_Hg11B, 8) \
  X(L_Hg21W, 256) \
  X(L_Hg21B, 16) \
  X(L_Hg31W, 256) \
  X(L_Hg31B, 16) \
  X(L_Hg41W, 256) \
  X(L_Hg41B, 16) \
  X(L_Hg51W, 1024) \
  X(L_Hg51B, 32) \
  X(L_Hg61W, 1024) \
  X(L_Hg61B, 32) \
  X(L_Hg71W, 1024) \
  X(L_Hg71B, 32) \
  X(L_Hg81W, 1024) \
  X(L_Hg81B, 32) \
  X(LDSE01W, 64) \
  X(LDSE02W, 24) \
  X(LDSE11W, 64) \
  X(LDSE12W, 24) \
  X(LDSE21W, 64) \
  X(LDSE22W, 24) \
  X(LDSE31W, 64) \
  X(LDSE32W, 24) \
  X(LSE01W, 64) \
  X(LSE02W, 24) \
  X(LSE11W, 64) \
  X(LSE12W, 24) \
  X(LSE21W, 64) \
  X(LSE22W, 24) \
  X(LSE31W, 64) \
  X(LSE32W, 24) \
  X(LSE41W, 64) \
  X(LSE42W, 24) \
  X(LSE51W, 64) \
  X(LSE52W, 24) \
  X(LSE61W, 64) \
  X(LSE62W, 24) \
  X(LSE71W, 64) \
  X(LSE72W, 24) \
  X(LSEFin1W, 1200) \
  X(LSEFin2W, 96) \
  X(LGGSW, 24) \
  X(LGGSB, 8) \
  X(LC0W, 16384) \
  X(LC0B, 128) \
  X(LC1W, 8192) \
  X(LC1B, 64) \
  X(LC2W, 2048) \
  X(LC2B, 32) \
  X(LXW, 512) \
  X(LXB, 16) \
  X(LX0W, 256) \
  X(LX0B, 16) \
  X(LX1W, 256) \
  X(LX1B, 16) \
  X(LX2W, 256) \
  X(LX2B, 16) \
  X(LX3W, 256) \
  X(LX3B, 16) \
  X(LX4W, 256) \
  X(LX4B, 16) \
  X(LX5W, 256) \
  X(LX5B, 16) \
  X(LX6W, 256) \
  X(LX6B, 16) \
  X(LX7W, 256) \
  X(LX7B, 16) \
  X(LX8W, 256) \
  X(LX8B, 16) \
  X(LX9W, 256) \
  X(LX9B, 16) \
  X(LX10W, 256) \
  X(LX10B, 16) \
  X(LX11W, 256) \
  X(LX11B, 16) \
  X(LX12W, 16) \
  X(LX12B, 1) \
  /* end */

enum mr_weight_id {
#define MR_W_ENUM(name, n) MR_W_##name,
  MR_WEIGHT_LIST(MR_W_ENUM)
#undef MR_W_ENUM
  MR_W_COUNT
};

/* Number of fp32 values in a complete blob. */
#define MR_WEIGHT_TOTAL 49673
/* Number of weight arrays in the blob. */
#define MR_WEIGHT_ARRAYS 146
/* 160 stencil directions (x, y, z) of the 192-point multi-scale descriptor. */
#define MR_STENCIL_POINTS 160

#endif
