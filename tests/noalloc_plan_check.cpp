// Host-only check of noalloc_plan, the launch plan of
// wn_forward_fp64_device_noalloc: for every size and SM count the face-split
// partial sums (nsplit x nq doubles) fit the library's fixed scratch array, the
// splits cover every face, and on a large SM count with few queries the cap
// actually engages (the uncapped plan would not fit). Built and run by
// tests/test_capi.py against libwn_b200.so; needs no GPU. Prints "ok" on success.
#include <cstdio>

#include "wn_internal.h"

int main() {
  const int sms_list[] = {1, 148, 1024, 4096};
  const long long nq_list[] = {1, 7, 100, 1000, 4096, 40000, 1 << 19};
  const long long nf_list[] = {1, 100, 20480, 327680, 5242880};
  int capped = 0;
  for (int sms : sms_list)
    for (long long nq : nq_list)
      for (long long nf : nf_list) {
        const wn::Fp64Plan p = wn::noalloc_plan(nf, nq, sms);
        const long long cap = wn::kNoAllocScratchDoubles / nq;
        if (p.nsplit < 1 || p.nsplit > (cap > 0 ? cap : 1) ||
            (p.nsplit > 1 && p.scratch_doubles != p.nsplit * nq) ||
            p.scratch_doubles > wn::kNoAllocScratchDoubles || p.f_chunk * p.nsplit < nf) {
          std::printf("bad plan: sms %d nq %lld nf %lld nsplit %lld f_chunk %lld scratch %lld\n",
                      sms, nq, nf, static_cast<long long>(p.nsplit),
                      static_cast<long long>(p.f_chunk), static_cast<long long>(p.scratch_doubles));
          return 1;
        }
        if (wn::plan_fp64(nf, nq, sms).scratch_doubles > wn::kNoAllocScratchDoubles) ++capped;
      }
  if (capped == 0) {
    std::printf("the cap never engaged\n");
    return 1;
  }
  std::printf("ok %d capped plans\n", capped);
  return 0;
}
