/*
 * constants.h -- compile-time limits shared by the drop-in graph API.
 *
 * Same names and values as the reference's src/constants.h:9-41 so that
 * callers written against the reference (the BIF/XMLBIF parsers, the
 * benchmark drivers, example-belief-propagation.c) compile unchanged.
 *
 * What differs in this library (documented, not a source-level change):
 *  - MAX_DEGREE is kept for source compatibility only.  The reference
 *    asserts a node has at most MAX_DEGREE in- and out-edges (graph.c:184,
 *    :201); this library stores edges in CSR arrays built by a stable
 *    counting sort and has no per-node cap.
 *  - BLOCK_SIZE*, WARP_SIZE and BATCH_SIZE describe the reference's own
 *    sm_35 launch shapes and OpenACC batch; the sm_100a kernels here size
 *    their grids themselves.  BATCH_SIZE is still the delta-check period of
 *    the *_acc propagate entry points.
 */

#ifndef CONSTANTS_H_
#define CONSTANTS_H_

#define CHAR_BUFFER_SIZE 50

#define MAX_STATES 10

#define DEFAULT_STATE 1.0

#define WEIGHT_INFINITY 99999

#define BATCH_SIZE 10

#define NUM_ITERATIONS 200

#define PRECISION 1E-3f

#define BLOCK_SIZE 1024

#define BLOCK_SIZE_2_D_X 64

#define BLOCK_SIZE_2_D_Y 16

#define BLOCK_SIZE_3_D_X 4

#define BLOCK_SIZE_3_D_Y 16

#define BLOCK_SIZE_3_D_Z 16

#define MAX_NUM_NODES 1048

#define WARP_SIZE 32

#define MAX_DEGREE 20

#define CHARS_IN_KEY 20

#endif /* CONSTANTS_H_ */
