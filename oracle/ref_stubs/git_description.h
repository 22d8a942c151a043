/* Stand-in for the generated git_description.h of the reference build. */
#ifndef GIT_DESCRIPTION
#define GIT_DESCRIPTION "oracle-build"
#endif
