// Test infrastructure only: the Cactus table utilities that
// AsterX/src/estimate_error.hxx names (group tag and centering tables of the
// regrid variables).  The checker passes the variables directly, so these
// are declared for compilation and never called.
#ifndef AXREF_SHIM_UTIL_TABLE_H
#define AXREF_SHIM_UTIL_TABLE_H

#define UTIL_ERROR_TABLE_NO_SUCH_KEY (-4)

int CCTK_GroupTagsTableI(int group);
int CCTK_GroupCenteringTableI(int group);
int Util_TableGetIntArray(int handle, int nvalues, int *array, const char *key);

#endif
