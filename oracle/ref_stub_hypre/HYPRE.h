/* Stand-in for a HYPRE header (oracle test infrastructure): everything the
 * reference's HypreFDM 3D solver uses is in _hypre_utilities.h. */
#include "_hypre_utilities.h"
