/* Single-process stand-in for the few MPI calls the MG-alphaGCD sources make
 * (oracle test infrastructure: lets the reference build into oracle/_ref/). */
#pragma once
#include <time.h>
typedef int MPI_Comm;
typedef int MPI_Info;
#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_COMM_TYPE_SHARED 0
#define MPI_SUCCESS 0
#define MPI_MAX_ERROR_STRING 64
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Comm_split_type(MPI_Comm, int, int, MPI_Info, MPI_Comm *c) { *c = 0; return 0; }
static inline int MPI_Comm_free(MPI_Comm *) { return 0; }
static inline int MPI_Error_string(int, char *s, int *l) { s[0] = 0; *l = 0; return 0; }
static inline double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
