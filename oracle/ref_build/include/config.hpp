/* Hand-written configuration header for building the reference library's
 * twisted-mass hot path as a single-rank, OpenMP, CPU-layout oracle.
 * Stands in for the autotools-generated config.hpp (configure.ac:5-494). */
#ifndef _ORACLE_REF_CONFIG_HPP
#define _ORACLE_REF_CONFIG_HPP

#define CONFIG_FLAGS "oracle-ref single-rank openmp"
#define CONFIG_TIME "oracle-ref"
#define CAN_DEMANGLE 0
#define USE_MPI 1
#define HAVE_OPENMP 1
#define NO_THREADS 0
#define OPENMP_THREADS 1
#define CUDA_THREADS 2
#define THREADS_TYPE OPENMP_THREADS
#define CUDA_MANAGED
#define CUDA_HOST_AND_DEVICE
#define CUDA_DEVICE
#define DEFAULT_MEMORY_LAYOUT CPU
#define IS_LITTLE_ENDIAN (__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__)
#define NATIVE_HIGH_PREC 0
#define GMP_HIGH_PREC 1
#define HIGH_PREC_TYPE NATIVE_HIGH_PREC
#define MAX_VERBOSITY_LV 3
#define NDIM 4
#define _ASM_BOOKMARK_SYMBOL "#"

#define _CONCAT(X,Y) X##Y
#define CONCAT(X,Y) _CONCAT(X,Y)
#define CONCAT2(s1,s2) CONCAT(s1,s2)
#define CONCAT3(s1,s2,s3) CONCAT(CONCAT2(s1,s2),s3)
#define NAME2(s1,s2) CONCAT3(s1,_,s2)
#define NAME3(s1,s2,s3) NAME2(CONCAT3(s1,_,s2),s3)
#define NAME4(s1,s2,s3,s4) NAME3(CONCAT3(s1,_,s2),s3,s4)
#define REORDER_BARRIER() __asm volatile ("")
#define MACRO_GUARD(...) do{__VA_ARGS__}while(0)
#define TO_STRING_INTERNAL(x) #x
#define TO_STRING(x) TO_STRING_INTERNAL(x)
#define LINE_AS_STRING TO_STRING(__LINE__)
#define ASM_BOOKMARK(COMMENT) __asm volatile ("")
#define ASM_BOOKMARK_BEGIN(COMMENT) ASM_BOOKMARK("BEGIN " COMMENT)
#define ASM_BOOKMARK_END(COMMENT) ASM_BOOKMARK("END " COMMENT)

#endif
