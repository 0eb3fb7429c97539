// evp_batch.h -- library-internal interface of a batch of solves (the serving loop's engine).
//
// A Batch owns one CUDA stream and one Engine.  Members join with add(): their deck is
// opened on the batch's stream and their first increment begins; every step() runs a
// few equilibrium iterations of all running members in batched launches, then, for each
// member whose iteration has stopped, the host side of the event: the end of the
// increment (rows, VTK, calc_c0) and the start of the next, or the end of the solve.
// Members advance independently (a member that converges starts its next increment while
// the others keep iterating); one that fails leaves with its status while the others go on.
#pragma once
#include "../../include/evp.h"
#include "evp_deck.h"

#include <string>

namespace evp {

class Batch;

Batch* batch_create();  // on the current device
void batch_destroy(Batch* b);
// Opens a member (deck already parsed into dk, moved from); returns its slot, or -1 with err set.
int batch_add(Batch* b, Deck&& dk, const std::string& fft_in, const std::string& out_dir, int mix, int modal, int flags,
              double deadline_s, std::string& err);
// Runs `rounds` rounds (each: a few iterations of every running member and the host side of
// their events).  Returns the number of members still running.
int batch_step(Batch* b, int rounds);
// 0 running, 1 finished (status in *status: 0 ok or a code), -1 no such slot.
int batch_slot(Batch* b, int slot, int* status, evp_report* rep, std::string* err);
void batch_remove(Batch* b, int slot);  // releases a finished slot's device memory
int batch_running(Batch* b);

}  // namespace evp
