/* Stand-in for MATLAB's mat.h (the reference includes it; it uses nothing
 * from it beyond matrix.h). */
#include "matrix.h"
