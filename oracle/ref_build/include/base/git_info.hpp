#ifndef _GIT_INFO
#define _GIT_INFO
 #define GIT_HASH "unknown"
 #define GIT_TIME "unknown"
 #define GIT_LOG "oracle build"
#endif
