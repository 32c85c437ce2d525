/*
 * b2e_adapter -- the drop-in hook between elegant's do_tracking() and the
 * engine's C ABI (include/elegant_b200.h).
 *
 * This file and b2e_adapter.c are written against elegant's own types
 * (ELEMENT_LIST, track.h:290-344; the element structures DRIFT, KQUAD, KSEXT,
 * CSBEND, CSRCSBEND, RFCA, ... track.h:1313-2528) and its parameter tables
 * (entity_description, track_data.c), so they compile inside elegant's tree.
 * A maintainer adds the call at the top of do_tracking() (do_tracking.c:144):
 *
 *   #ifdef HAVE_B2E
 *     if (!(flags & (TEST_PARTICLES | CLOSED_ORBIT_TRACKING | OPTIMIZING))) {
 *       double effort;
 *       long n_left = b2e_adapter_track(coord, *n_original, &beamline->elem, *P_central, n_passes,
 *                                       run->default_order, &effort, NULL, 0);
 *       if (n_left >= 0)
 *         return n_left;
 *     }
 *   #endif
 *
 * and links libelegant_b200.so.  A line the engine cannot take (an element
 * type outside its set, or a parameter set away from the default of
 * elegant's table where the engine has no slot for it) returns -1 before
 * anything is changed, and do_tracking goes on as it would without the hook.
 */
#ifndef B2E_ADAPTER_H
#define B2E_ADAPTER_H

/* Tracks np rows of coord (elegant's particle array: x, xp, y, yp, s,
 * delta, particleID, lossPass, ...) through the line that starts at `first`
 * for n_passes passes on the GPU.  On success returns the survivors n_left:
 * rows [0, n_left) hold them, rows [n_left, np) the lost particles with
 * their loss pass in column lossPassIndex, as do_tracking leaves them; a
 * lost row's coordinates are those at its loss (elegant also writes the
 * loss position and momentum there).  *effort, if not NULL, receives the
 * particle-passes (do_tracking.c:2758-2764).  Returns -1 with a reason in
 * why (if not NULL) when the line cannot be handed over, -2 when the engine
 * reported an error. */
long b2e_adapter_track(double **coord, long np, ELEMENT_LIST *first, double P_central, long n_passes,
                       long default_order, double *effort, char *why, long why_len);

/* Releases the engine context the adapter keeps between calls. */
void b2e_adapter_release(void);

#endif
