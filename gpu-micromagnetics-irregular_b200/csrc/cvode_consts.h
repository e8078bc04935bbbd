// cvode_consts.h — CVODE's default constants and internal flags, shared by
// the host-driven integrator (integrator.cu) and its device-resident form
// (integrator_dev.cu).  Values as published with CVODE (Hindmarsh et al.,
// ACM TOMS 31(3) 2005; cvode.c / cvode_nls.c / cvode_ls.c defaults), so the
// step sequence matches a CVODE run.
#pragma once
#include <float.h>

namespace {
constexpr int QMAXL = 5;
constexpr int MAXLL = 16;
constexpr double UROUND = DBL_EPSILON;
constexpr double FUZZ_FACTOR = 100.0, HLB_FACTOR = 100.0, HUB_FACTOR = 0.1, H_BIAS = 0.5;
constexpr int MAX_ITERS = 4;
constexpr double CORTES = 0.1, THRESH = 1.5, ETAMX1 = 10000.0, ETAMX2 = 10.0, ETAMX3 = 10.0;
constexpr double ETAMXF = 0.2, ETAMIN = 0.1, ETACF = 0.25, ADDON = 1.0e-6;
constexpr double BIAS1 = 6.0, BIAS2 = 6.0, BIAS3 = 10.0, ONEPSM = 1.000001;
constexpr int SMALL_NST = 10, MXNCF = 10, MXNEF = 7, MXNEF1 = 3, SMALL_NEF = 2, LONG_WAIT = 10;
constexpr int NLS_MAXCOR = 3, MSBP = 20, LS_MSBJ = 51;
constexpr double CRDOWN = 0.3, DGMAX = 0.3, RDIV = 2.0, LS_EPLIN = 0.05, LS_DGMAX = 0.2, GS_FACTOR = 1000.0;
constexpr int FIRST_CALL = 0, PREV_CONV_FAIL = 1, PREV_ERR_FAIL = 2, DO_ERROR_TEST = 3, PREDICT_AGAIN = 4,
              TRY_AGAIN = 5;
constexpr int NLS_CONTINUE = 901, NLS_CONV_RECVR = 902;
constexpr int CV_NO_FAILURES = 0, CV_FAIL_BAD_J = 1, CV_FAIL_OTHER = 2;
constexpr int LS_SUCCESS = 0, LS_RES_REDUCED = 1, LS_CONV_FAIL = 2, LS_QRSOL_FAIL = 3;
constexpr int SLOT_A = 0, SLOT_DOTS = 8;

}  // namespace
