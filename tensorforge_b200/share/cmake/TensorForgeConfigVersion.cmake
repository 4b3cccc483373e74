# Version check of tensorforge_b200's CMake package: the version is the package's VERSION
# file; only an exact match of a requested version is accepted (as the reference does).
file(READ "${CMAKE_CURRENT_LIST_DIR}/../../VERSION" PACKAGE_VERSION)
string(STRIP "${PACKAGE_VERSION}" PACKAGE_VERSION)
if(NOT PACKAGE_FIND_VERSION OR PACKAGE_VERSION VERSION_EQUAL PACKAGE_FIND_VERSION)
  set(PACKAGE_VERSION_COMPATIBLE TRUE)
  if(PACKAGE_VERSION VERSION_EQUAL PACKAGE_FIND_VERSION)
    set(PACKAGE_VERSION_EXACT TRUE)
  endif()
else()
  set(PACKAGE_VERSION_COMPATIBLE FALSE)
endif()
