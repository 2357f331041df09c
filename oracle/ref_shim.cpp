/*
 * ref_shim.cpp -- C entry points over the reference's own C++ SpikeContainer
 * (brian/utils/ccircular/circular.cpp, compiled from the reference tree by
 * oracle/build.py into oracle/_ref/).  TEST INFRASTRUCTURE ONLY: the tests
 * use it to pin the spike-history semantics (push, get_spikes with a
 * subgroup origin, LS[i:j] slices) that the oracle and the device ring
 * restate.  The reference sources are compiled where they lie; nothing of
 * them is copied here.
 */
#include "ccircular.h"
#include <cstring>

extern "C" {

void *ref_sc_create(int m) { return new SpikeContainer(m); }
void ref_sc_destroy(void *h) { delete (SpikeContainer *)h; }
void ref_sc_push(void *h, const long *x, int n) {
    ((SpikeContainer *)h)->push(const_cast<long *>(x), n);
}
/* neurons that spiked `delay` steps ago within [origin, origin+N), minus origin */
int ref_sc_get_spikes(void *h, int delay, int origin, int N, long *out, int cap) {
    long *r = nullptr; int n = 0;
    ((SpikeContainer *)h)->get_spikes(&r, &n, delay, origin, N);
    int k = n < cap ? n : cap;
    if (k > 0) std::memcpy(out, r, sizeof(long) * k);
    return n;
}
/* LS[i:j]: spikes of bins i..j-1 (0 = current step) */
int ref_sc_getslice(void *h, int i, int j, long *out, int cap) {
    long *r = nullptr; int n = 0;
    ((SpikeContainer *)h)->__getslice__(&r, &n, i, j);
    int k = n < cap ? n : cap;
    if (k > 0) std::memcpy(out, r, sizeof(long) * k);
    return n;
}

}
