# CMake package "tapp" for the B200 library, in place of the reference's
# installed package (its cmake/tapp-config.cmake.in): the same package name,
# components and imported targets, so that a consumer that does
#   find_package(tapp REQUIRED COMPONENTS reference)
#   target_link_libraries(app PRIVATE tapp::reference)
# links against lib/libtapp-b200.so instead when tapp_DIR points here.
#
#   tapp::api        INTERFACE: the TAPP headers (include/)
#   tapp::reference  SHARED IMPORTED: the library, with tapp::api
#
# Nothing is installed: the targets point into the source tree, where
# `make -C reference-implementation_b200` builds the library.

get_filename_component(_tapp_b200_pkg "${CMAKE_CURRENT_LIST_DIR}/.." ABSOLUTE)
get_filename_component(_tapp_b200_root "${_tapp_b200_pkg}/.." ABSOLUTE)
set(_tapp_b200_lib "${_tapp_b200_pkg}/lib/libtapp-b200.so")

set(tapp_VERSION "0.5.0")

if(NOT TARGET tapp::api)
  add_library(tapp::api INTERFACE IMPORTED)
  set_target_properties(tapp::api PROPERTIES
    INTERFACE_INCLUDE_DIRECTORIES "${_tapp_b200_root}/include")
endif()

if(NOT TARGET tapp::reference AND EXISTS "${_tapp_b200_lib}")
  add_library(tapp::reference SHARED IMPORTED)
  set_target_properties(tapp::reference PROPERTIES
    IMPORTED_LOCATION "${_tapp_b200_lib}"
    IMPORTED_NO_SONAME TRUE
    INTERFACE_LINK_LIBRARIES tapp::api)
endif()

# components: api and reference; none requested means every one present
set(_tapp_components api reference)
if(NOT tapp_FIND_COMPONENTS)
  foreach(_c IN LISTS _tapp_components)
    if(TARGET tapp::${_c})
      list(APPEND tapp_FIND_COMPONENTS ${_c})
    endif()
  endforeach()
endif()
set(tapp_FOUND TRUE)
foreach(_c IN LISTS tapp_FIND_COMPONENTS)
  if(_c IN_LIST _tapp_components AND TARGET tapp::${_c})
    set(tapp_${_c}_FOUND TRUE)
  else()
    set(tapp_${_c}_FOUND FALSE)
    if(tapp_FIND_REQUIRED_${_c})
      set(tapp_FOUND FALSE)
      if(_c IN_LIST _tapp_components)
        set(tapp_NOT_FOUND_MESSAGE "tapp component '${_c}' not found (build ${_tapp_b200_lib} first)")
      else()
        set(tapp_NOT_FOUND_MESSAGE "tapp: unknown component '${_c}' requested")
      endif()
    endif()
  endif()
endforeach()
