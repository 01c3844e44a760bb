// Host-only stand-ins for the reference's device-qualifier macros, so that its
// pure host/device math headers compile with g++ in this container.  Used only
// by oracle/ref_probe (a test-time cross-check), never by the product.
#pragma once
#define COLLECTION_GLOBAL
#define COLLECTION_SIMT_DEVICE inline
#define COLLECTION_HOST inline
#define COLLECTION_HOST_DEVICE inline
#define COLLECTION_AIV_GLOBAL
#define COLLECTION_SIMT_VF
#define __gm__
