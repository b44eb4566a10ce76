/* Fallback for the undeclared multigrid-level name used in one diagnostic
 * message of the reference's residual monitor (one grid level in the oracle). */
static const int level = 0;
