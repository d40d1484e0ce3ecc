/* bbb_restart.c -- the reference's restart file, written and read from the
 * library's host state.
 *
 * The file is the raw sequence that out_restart / in_restart of
 * src/domain.c:3223-3413 write and read (a file format, so the same bytes):
 *   ttime, dt0, dt (real), stepnum, rec_paraview_stepnum_out (int);
 *   for u, v, w on Gfx, Gfy, Gfz (s3b reals each): the field, its previous
 *     step, the diffusion history (only when the step is explicit: the
 *     reference omits it when built with -DIMPLICIT), the advection
 *     history, diffusion, advection, the intermediate velocity;
 *   p, phi, p0 (Gcc reals); phase, phase_shell (Gcc ints);
 *   flag_u, flag_v, flag_w (Gfx/Gfy/Gfz ints); bc_plane_pos[9];
 *   parts (nparts part_struct records); coeff_stride (int);
 *   the 18 Lamb coefficient arrays (nparts * coeff_stride reals each:
 *     p, phi, chi; re, im; current, previous, the one before);
 *   the recorder clocks (flow field, ParaView, particle, restart,
 *     precursor), pid_int, pid_back;
 *   gradP.z and the member after it (the reference writes two reals from
 *   &gradP.z, src/domain.c:3310, and reads one back, :3412).
 * The explicit/implicit choice follows the run-time option
 * `implicit` where the reference fixes it at compile time.  The arrays are
 * the host copies: pull the device state first (cuda_dom_pull,
 * cuda_part_pull), and push after reading (cuda_dom_push, cuda_part_push),
 * the order src/bluebottle.c:454-470 and :786-791 use. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "../../include/bluebottle_b200.h"

#define WEAK __attribute__((weak))

/* recorder state the file carries (defined by src/bluebottle.c in the
 * reference's own program; weak here like every shared global) */
WEAK int rec_paraview_stepnum_out;
WEAK real rec_flow_field_ttime_out, rec_paraview_ttime_out,
  rec_particle_ttime_out, rec_restart_ttime_out, rec_prec_ttime_out;
WEAK real bc_plane_pos[9];

/* the rest of src/bluebottle.c's globals that the reference's own host
 * files (src/domain.c, src/particle.c, src/vtk.c) read: the other
 * recorder counters and the precursor's inflow planes and forcing
 * (src/bluebottle.h:1118-1281, 1653-1791, 2347-2360).  With them those
 * files link against this library unchanged; the library itself only
 * carries them. */
WEAK int rec_flow_field_stepnum_out, rec_prec_stepnum_out,
  rec_particle_stepnum_out;
WEAK real rec_prec_flow_field_ttime_out;
WEAK real *u_WE, *u_SN_S, *u_SN_N, *u_BT_B, *u_BT_T;
WEAK real *v_WE_W, *v_WE_E, *v_SN, *v_BT_B, *v_BT_T;
WEAK real *w_WE_W, *w_WE_E, *w_SN_S, *w_SN_N, *w_BT;
WEAK real turbA, turbl;

extern bbb_options g_opt;
void bbb_set_status(int status, const char *where);

/* one contiguous run of the file */
typedef struct {
  void *ptr;
  size_t esz;
  long long count;
} rs_item;

#define RS_MAX 96

/* The file's runs in order; `writing` selects the writer's two reals at
 * the end instead of the reader's one.  Returns the number of runs. */
static int rs_layout(rs_item *it, int writing)
{
  int n = 0;
  long long fx = Dom.Gfx.s3b, fy = Dom.Gfy.s3b, fz = Dom.Gfz.s3b;
  long long cc = Dom.Gcc.s3b;
  long long nc = (long long)nparts * coeff_stride;
#define RS(p, e, c) do { it[n].ptr = (void *)(p); it[n].esz = (e); \
                         it[n].count = (c); n++; } while(0)
  RS(&ttime, sizeof(real), 1);
  RS(&dt0, sizeof(real), 1);
  RS(&dt, sizeof(real), 1);
  RS(&stepnum, sizeof(int), 1);
  RS(&rec_paraview_stepnum_out, sizeof(int), 1);
  {
    real *vel[3] = {u, v, w}, *vel0[3] = {u0, v0, w0};
    real *d0[3] = {diff0_u, diff0_v, diff0_w}, *c0[3] = {conv0_u, conv0_v, conv0_w};
    real *df[3] = {diff_u, diff_v, diff_w}, *cv[3] = {conv_u, conv_v, conv_w};
    real *st[3] = {u_star, v_star, w_star};
    long long len[3] = {fx, fy, fz};
    for(int a = 0; a < 3; a++) {
      RS(vel[a], sizeof(real), len[a]);
      RS(vel0[a], sizeof(real), len[a]);
      if(!g_opt.implicit) RS(d0[a], sizeof(real), len[a]);
      RS(c0[a], sizeof(real), len[a]);
      RS(df[a], sizeof(real), len[a]);
      RS(cv[a], sizeof(real), len[a]);
      RS(st[a], sizeof(real), len[a]);
    }
  }
  RS(p, sizeof(real), cc);
  RS(phi, sizeof(real), cc);
  RS(p0, sizeof(real), cc);
  RS(phase, sizeof(int), cc);
  RS(phase_shell, sizeof(int), cc);
  RS(flag_u, sizeof(int), fx);
  RS(flag_v, sizeof(int), fy);
  RS(flag_w, sizeof(int), fz);
  RS(bc_plane_pos, sizeof(real), 9);
  RS(parts, sizeof(part_struct), nparts);
  RS(&coeff_stride, sizeof(int), 1);
  {
    real *cf[18] = {pnm_re, pnm_im, pnm_re0, pnm_im0, pnm_re00, pnm_im00,
      phinm_re, phinm_im, phinm_re0, phinm_im0, phinm_re00, phinm_im00,
      chinm_re, chinm_im, chinm_re0, chinm_im0, chinm_re00, chinm_im00};
    for(int a = 0; a < 18; a++) RS(cf[a], sizeof(real), nc);
  }
  RS(&rec_flow_field_ttime_out, sizeof(real), 1);
  RS(&rec_paraview_ttime_out, sizeof(real), 1);
  RS(&rec_particle_ttime_out, sizeof(real), 1);
  RS(&rec_restart_ttime_out, sizeof(real), 1);
  RS(&rec_prec_ttime_out, sizeof(real), 1);
  RS(&pid_int, sizeof(real), 1);
  RS(&pid_back, sizeof(real), 1);
  RS(&gradP.z, sizeof(real), 1);
  if(writing) RS(&gradP.zm, sizeof(real), 1);
#undef RS
  return n;
}

static const char *rs_path(const char *path, char *buf, size_t len)
{
  if(path && path[0]) return path;
  snprintf(buf, len, "./input/restart.config");
  return buf;
}

/* src/domain.c:3223 out_restart */
int bbb_out_restart(const char *path)
{
  char buf[1024];
  rs_item it[RS_MAX];
  if(!Dom.Gcc.s3b || !u || !p) {
    bbb_set_status(BBB_ERR_STATE, "out_restart before domain_init");
    return BBB_ERR_STATE;
  }
  const char *fn = rs_path(path, buf, sizeof(buf));
  FILE *f = fopen(fn, "wb");
  if(!f) {
    bbb_set_status(BBB_ERR_CONFIG, "out_restart: cannot create the file");
    return BBB_ERR_CONFIG;
  }
  int n = rs_layout(it, 1), ok = 1;
  for(int a = 0; a < n && ok; a++) {
    if(it[a].count <= 0) continue;
    if(!it[a].ptr) { ok = 0; break; }
    ok = fwrite(it[a].ptr, it[a].esz, (size_t)it[a].count, f) == (size_t)it[a].count;
  }
  if(fclose(f) != 0) ok = 0;
  if(!ok) {
    bbb_set_status(BBB_ERR_CONFIG, "out_restart: write failed");
    return BBB_ERR_CONFIG;
  }
  return BBB_OK;
}

/* src/domain.c:3318 in_restart: the domain and particles must be set up
 * from the same input files first (array sizes come from them) */
int bbb_in_restart(const char *path)
{
  char buf[1024];
  rs_item it[RS_MAX];
  if(!Dom.Gcc.s3b || !u || !p) {
    bbb_set_status(BBB_ERR_STATE, "in_restart before domain_init");
    return BBB_ERR_STATE;
  }
  const char *fn = rs_path(path, buf, sizeof(buf));
  FILE *f = fopen(fn, "rb");
  if(!f) {
    bbb_set_status(BBB_ERR_CONFIG, "in_restart: cannot open the file");
    return BBB_ERR_CONFIG;
  }
  int saved_stride = coeff_stride;
  int n = rs_layout(it, 0), ok = 1;
  for(int a = 0; a < n && ok; a++) {
    if(it[a].count <= 0) continue;
    if(!it[a].ptr) { ok = 0; break; }
    ok = fread(it[a].ptr, it[a].esz, (size_t)it[a].count, f) == (size_t)it[a].count;
    /* the coefficient arrays were sized by the set-up's stride */
    if(ok && it[a].ptr == (void *)&coeff_stride && coeff_stride != saved_stride) {
      coeff_stride = saved_stride;
      ok = 0;
    }
  }
  fclose(f);
  if(!ok) {
    bbb_set_status(BBB_ERR_CONFIG, "in_restart: short or mismatched file");
    return BBB_ERR_CONFIG;
  }
  return BBB_OK;
}
