// Stand-in for the CMake-generated version header of the reference build.
#define GIT_REV "oracle-shim"
#define GIT_TAG "N/A"
#define GIT_BRANCH "N/A"
