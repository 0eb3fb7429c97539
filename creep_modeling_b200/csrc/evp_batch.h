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

Batch* batch_create(int priority = 0);  // on the current device; priority: its stream's CUDA priority
// The highest stream priority of the device (numerically smallest); *lowest gets the lowest.
int batch_priority_range(int* lowest);
void batch_destroy(Batch* b);
// Opens a member (deck already parsed into dk, moved from); returns its slot, or -1 with err set.
int batch_add(Batch* b, Deck&& dk, const std::string& fft_in, const std::string& out_dir, int mix, int modal, int flags,
              double deadline_s, std::string& err);
// Runs `rounds` rounds (each: a few iterations of every running member and the host side of
// their events).  Returns the number of members still running.
int batch_step(Batch* b, int rounds);
// The same round in three calls, so that one host thread can keep several batches (on
// streams of different priority) busy: batch_launch queues a round (false when no member
// runs), batch_ready says whether its iterations have run, batch_finish does the host side
// of the round's events and returns the number of members still running.
bool batch_launch(Batch* b);
bool batch_ready(Batch* b);
int batch_finish(Batch* b);
// 0 running, 1 finished (status in *status: 0 ok or a code), -1 no such slot.
int batch_slot(Batch* b, int slot, int* status, evp_report* rep, std::string* err);
void batch_remove(Batch* b, int slot);  // releases a finished slot's device memory
int batch_running(Batch* b);

}  // namespace evp
