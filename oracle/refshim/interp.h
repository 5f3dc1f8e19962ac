/* Empty stand-in for libEM/interp.h (nothing from it is used by the
 * inserters compiled in oracle/build_ref.sh). TEST INFRASTRUCTURE ONLY. */
