/* Status codes written to every `ierr` argument.  Same values, in the same
 * order, as hmat_lib include/hmat_lib/error.h:9-16. */
#ifndef HODLR_ERROR_H
#define HODLR_ERROR_H

enum ErrorCode {
  SUCCESS,
  ALLOCATION_FAILURE,
  SVD_FAILURE,
  SVD_ALLOCATION_FAILURE,
  INPUT_ERROR,
  QR_FAILURE
};

#endif
