/* Largest off-diagonal rank in the tree (hmat_lib src/utils.c:5). */
#ifndef _HODLR_UTILS_MAIN
#define _HODLR_UTILS_MAIN

#ifdef __cplusplus
extern "C" {
#endif

struct TreeHODLR;

int get_highest_s(const struct TreeHODLR *const hodlr);

#ifdef __cplusplus
}
#endif

#endif
