// Internal interface between the serving loop (server.cu) and the batched group engine
// (group.cuh, compiled in ssfft.cu's translation unit).  Not part of the C ABI.
#pragma once

#include <stddef.h>

#include <string>
#include <vector>

#include "../../include/ssfft.h"

// A request as the server holds it: its arrays copied at submission.
struct GroupJob {
  ssfft_request req;
  std::vector<double> rotations;
  std::vector<int32_t> orient, phase;
  double submit_time;
  size_t bytes;
};

// Slot states of a group (GroupCtl::state).
enum { GS_EMPTY = 0, GS_FRESH = 1, GS_SOLVE = 2, GS_DONE = 3, GS_FAILED = 4 };

struct Group;
Group *group_new();
void group_delete(Group *g);
int group_init(Group *g, const ssfft_config &cfg, int slots, bool voxel, bool rates, int dev);
int group_load(Group *g, int s, const GroupJob &j);
int group_run(Group *g);
int group_slot_state(Group *g, int s);
void group_slot_result(Group *g, int s, ssfft_solve_out *o);
int group_read_stress(Group *g, int s, double *dst);
int group_release_slot(Group *g, int s);
long long group_launches(Group *g);
// Ask the group's running launch to return at its next pass boundary (any thread), and
// clear that request (the group's driver thread, before it runs the group again).
void group_wake(Group *g);
void group_clear_wake(Group *g);
