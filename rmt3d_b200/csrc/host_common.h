// Shared host-side helpers: thread-local error message and status plumbing.
#pragma once
#include <cstddef>
#include <string>
#include <vector>

#include "rmt3d_gpu.h"

struct rmt3d_scene;

namespace rmt3d {
int fail(int code, const std::string &msg);

// Graph-mode stepping split in two, for callers that keep many scenes in
// flight: queue nsteps step-graph launches on the scene's stream (building
// the graph first if needed), then wait and collect the outcome as
// rmt3d_run does.  Scenes in profiling or eager mode run eagerly in
// steps_launch and steps_finish only reports.
int steps_launch(rmt3d_scene *s, int nsteps);
int steps_finish(rmt3d_scene *s, int *status);

// Equally sized scenes (same grid, form and multigrid schedule, all prepared)
// stepped together by one graph: per-scene phases as parallel branches, each
// multigrid solve one batched solve over the group.  group_finish fills one
// status per scene.
struct scene_group;
int group_create(rmt3d_scene *const *scenes, int n, scene_group **out);
// a scene's multigrid schedule, as groups must share it: v_down, v_up,
// smoother mode, cluster launch, cluster coarse sub-cycle's largest level
void scene_schedule(rmt3d_scene *s, int out[5]);
int group_launch(scene_group *g, int nsteps);
int group_finish(scene_group *g, int *status);
// true once the group's launched steps have all run (group_finish then
// returns without waiting)
bool group_done(scene_group *g);
void group_destroy(scene_group *g);
long long group_mg_launches(const scene_group *g);

// Checkpoint files (files.cc).  A packed checkpoint holds kChkFields
// fields in kChkNames order, each nslices slices of slice_len doubles.
constexpr int kChkFields = 8;
extern const char *const kChkNames[kChkFields];
int chk_make_dir(const char *dir);
int chk_write_files(const char *dir, const double *buf, size_t slice_len, int nslices, int compress);
// *status: 0 read, 1 a file missing, 2 a file empty (the reference's codes)
int chk_read_files(const char *dir, double *buf, size_t slice_len, int nslices, int *status);
int chk_write_recover_cfg(const char *dir, const rmt3d_scene_desc &d, double dt);
// a slice u[a + d1 b] in write_slice's format 0, 1 or 2; c1, c2 are the
// coordinates of the two axes, m the x extent written in the gnuplot header
int slice_write_file(const char *filename, const double *u, int d1, int d2, int format, const double *c1,
                     const double *c2, int m);
// tracer files: binary (count, then float x y z per tracer) or text lines
int tracer_write_file(const char *filename, const float *pos, int n, int binary);
int tracer_read_file(const char *filename, int n, std::vector<float> &pos);
}
