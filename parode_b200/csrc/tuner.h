// tuner.h -- measured choice of the block-response leaf's block length.
//
// The block length B = 2^R of the response leaf trades the window GEMMs'
// work (growing with B) against the carry over blocks (shrinking with B) and
// the FP64 build of W's tables.  The engines pick R with a cost model
// (response_log2_block); ParODE_TuneResponseBlock times the candidates on the
// device for a class of systems instead and stores the fastest here, and
// every plan or batch made afterwards for a system of that class uses it.
// The table can be saved and loaded per GPU (one entry per line).
#pragma once

#include <string>

namespace parode {

// A class of systems: solver, padded scan dimension (power of two), input
// and output counts (powers of two), horizon (log2 of the scan steps,
// rounded up) and precision form.
struct TuneClass {
    int solver = 0, np = 0, m = 0, p = 0, tclass = 0, precision = 0;
};

TuneClass tune_class(int solver, int Ns, int m, int p, long nScan, int precision);
// The measured log2 block length of the class, or -1 when it was not tuned.
int tuned_log2_block(const TuneClass& c);
void tune_store(const TuneClass& c, int log2B, float ms);
void tune_clear();
// Text form: one line per entry, "gpu solver np m p tclass precision log2B ms";
// load keeps the entries of `gpu` and returns how many it read.
std::string tune_dump(const std::string& gpu);
int tune_load_text(const std::string& text, const std::string& gpu);

}  // namespace parode
