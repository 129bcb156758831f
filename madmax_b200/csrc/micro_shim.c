/*
 * micro_shim.c -- the micro side of the reference's macro-micro coupling,
 * served by the device-resident serving loop.
 *
 * The reference's micro process answers the macro's requests in a blocking
 * loop (micro/src/main.c:114-153) on message_t (inc/comm.h:18-27):
 * ACTION_MICRO_CALC_STRESS fills stress_ave from strain_mac,
 * ACTION_MICRO_CALC_C_TANGENT fills c_tangent_ave, ACTION_MICRO_CALC_RHO
 * fills rho (a constant, 1e7: micro/src/init.c:9), ACTION_MICRO_END ends the
 * loop without a reply.  For linear materials the reference computes the
 * finite-difference tangent around zero strain once (micro/src/init.c:54-59)
 * and answers every stress request with C eps and every tangent request with
 * C (micro/src/homogenize.c:3-21, 35-49).  sp_micro does the same on one
 * geometry of an sp_server (SP_MICRO_LINEAR), or answers every request with
 * a serving-loop solve at the requested strain (SP_MICRO_SOLVE).  The
 * transport stays the caller's: sp_micro_serve takes receive and send
 * callbacks (an MPI program passes its comm_micro_recv / comm_micro_send).
 */
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include "sp_internal.h"

_Static_assert(sizeof(sp_message) == 400, "sp_message must match message_t");
_Static_assert(offsetof(sp_message, strain_mac) == 8, "sp_message layout");
_Static_assert(offsetof(sp_message, stress_ave) == 56, "sp_message layout");
_Static_assert(offsetof(sp_message, c_tangent_ave) == 104, "sp_message layout");
_Static_assert(offsetof(sp_message, rho) == 392, "sp_message layout");

struct sp_micro_s {
  sp_server *srv;
  int geom, mode, have_lin;
  double rho;
  double clin[36];
  double timeout_s;
  long long requests;
};

int sp_micro_create(sp_server *srv, int geometry, int mode, double rho, sp_micro **out) {
  if (!srv || !out) return sp_set_error(SP_ERR_ARG, "sp_micro_create: null argument");
  if (mode != SP_MICRO_LINEAR && mode != SP_MICRO_SOLVE)
    return sp_set_error(SP_ERR_ARG, "sp_micro_create: unknown mode");
  sp_micro *m = (sp_micro *)calloc(1, sizeof(*m));
  if (!m) return sp_set_error(SP_ERR_NOMEM, "sp_micro_create");
  m->srv = srv;
  m->geom = geometry;
  m->mode = mode;
  m->rho = rho;
  m->timeout_s = 600.0;
  *out = m;
  return SP_OK;
}

int sp_micro_destroy(sp_micro *m) {
  free(m);
  return SP_OK;
}

/* one serving-loop request: stress and FD tangent at eps */
static int request(sp_micro *m, const double *eps, double *stress, double *tangent) {
  int geom = m->geom;
  double t_arr = 0.0, t_done = 0.0;
  sp_solve_info info;
  int rc = sp_server_replay(m->srv, 1, &geom, eps, &t_arr, &t_done, stress, tangent, &info,
                            m->timeout_s);
  if (rc) return rc;
  m->requests++;
  if (info.status)
    return sp_set_error(SP_ERR_NOCONV, "micro request did not converge (relres %.3e)", info.relres);
  return SP_OK;
}

static int linear_tangent(sp_micro *m) {
  if (m->have_lin) return SP_OK;
  double zero[6] = {0, 0, 0, 0, 0, 0}, st[6];
  SP_TRY_C(request(m, zero, st, m->clin));
  m->have_lin = 1;
  return SP_OK;
}

int sp_micro_handle(sp_micro *m, sp_message *msg) {
  if (!m || !msg) return sp_set_error(SP_ERR_ARG, "sp_micro_handle: null argument");
  double tan[36], st[6];
  switch (msg->action) {
    case SP_ACTION_MICRO_CALC_STRESS:
    case SP_ACTION_MICRO_CALC_C_TANGENT:
      if (msg->num_voigt != 6)
        return sp_set_error(SP_ERR_ARG, "sp_micro_handle: num_voigt %d (3D needs 6)", msg->num_voigt);
      if (m->mode == SP_MICRO_LINEAR) {
        SP_TRY_C(linear_tangent(m));
        if (msg->action == SP_ACTION_MICRO_CALC_STRESS) {
          for (int i = 0; i < 6; i++) {
            double s = 0.0;
            for (int j = 0; j < 6; j++) s += m->clin[i * 6 + j] * msg->strain_mac[j];
            msg->stress_ave[i] = s;
          }
        } else {
          memcpy(msg->c_tangent_ave, m->clin, sizeof(m->clin));
        }
      } else {
        SP_TRY_C(request(m, msg->strain_mac, st, tan));
        if (msg->action == SP_ACTION_MICRO_CALC_STRESS)
          memcpy(msg->stress_ave, st, sizeof(st));
        else
          memcpy(msg->c_tangent_ave, tan, sizeof(tan));
      }
      return SP_OK;
    case SP_ACTION_MICRO_CALC_RHO:
      msg->rho = m->rho;
      return SP_OK;
    case SP_ACTION_MICRO_END:
      return SP_OK;
    default:
      return sp_set_error(SP_ERR_ARG, "sp_micro_handle: action %d not identified", msg->action);
  }
}

int sp_micro_serve(sp_micro *m, sp_message_recv recv, sp_message_send send, void *ctx,
                   long long *handled) {
  if (!m || !recv || !send) return sp_set_error(SP_ERR_ARG, "sp_micro_serve: null argument");
  sp_message msg;
  long long n = 0;
  memset(&msg, 0, sizeof(msg));
  while (msg.action != SP_ACTION_MICRO_END) {
    if (recv(&msg, ctx)) return sp_set_error(SP_ERR_STATE, "sp_micro_serve: receive failed");
    SP_TRY_C(sp_micro_handle(m, &msg));
    n++;
    if (handled) *handled = n;
    if (msg.action != SP_ACTION_MICRO_END && send(&msg, ctx))
      return sp_set_error(SP_ERR_STATE, "sp_micro_serve: send failed");
  }
  return SP_OK;
}

int sp_micro_requests(const sp_micro *m, long long *requests) {
  if (!m || !requests) return sp_set_error(SP_ERR_ARG, "sp_micro_requests: null argument");
  *requests = m->requests;
  return SP_OK;
}
