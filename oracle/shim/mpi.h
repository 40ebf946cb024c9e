/* Single-rank stand-in for the parts of the MPI API that the PGMG reference
 * library uses (common.hh:8 and every translation unit that includes it).
 *
 * TEST INFRASTRUCTURE ONLY: this header lets the unmodified reference sources
 * (buffer.cc common.cc geometry.cc region.cc region_tr.cc multigrid.cc) be
 * compiled into the CPU oracle library under oracle/_ref.  It is never part of
 * the product.
 *
 * Semantics (one process, rank 0, communicator size 1):
 *   - Cartesian communicators are 1x1x1; MPI_Cart_rank maps every (possibly
 *     periodic-wrapped) coordinate to rank 0 (geometry.cc:164-172 only asks for
 *     in-range or periodic neighbours).
 *   - Point-to-point messages go to self.  MPI_Isend copies the payload into
 *     an internal queue and completes at once; MPI_Irecv takes the first queued
 *     message with the same (tag, communicator) or registers a pending receive
 *     that a later send satisfies.  A wait on a receive that never matched
 *     aborts with a message (it would be a deadlock under real MPI).
 *   - Reductions and broadcasts over one rank are copies.
 * Written to compile under -ansi -pedantic (C++98), as the reference does
 * (config/config.mk.linux:8).
 */
#ifndef PGMG_ORACLE_MPI_SHIM_H
#define PGMG_ORACLE_MPI_SHIM_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <list>
#include <vector>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
struct MPI_Status { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; };
typedef int MPI_Request;

#define MPI_COMM_NULL (-1)
#define MPI_COMM_WORLD 0
#define MPI_UNDEFINED (-32766)
#define MPI_SUCCESS 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_FLOAT 3
#define MPI_UNSIGNED 4
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_STATUS_IGNORE ((MPI_Status*) 0)
#define MPI_STATUSES_IGNORE ((MPI_Status*) 0)
#define MPI_REQUEST_NULL 0

namespace pgmg_mpi_shim {

inline size_t type_size(MPI_Datatype t) {
	switch(t) {
		case MPI_DOUBLE: return sizeof(double);
		case MPI_FLOAT: return sizeof(float);
		case MPI_INT: return sizeof(int);
		case MPI_UNSIGNED: return sizeof(unsigned int);
	}
	fprintf(stderr,"mpi shim: unknown datatype %d\n",t);
	abort();
	return 0;
}

struct message {
	int tag;
	MPI_Comm comm;
	std::vector<char> payload;
};

struct pending_recv {
	int id;
	int tag;
	MPI_Comm comm;
	void *buf;
	size_t cap;
};

struct state {
	std::list<message> queue;
	std::list<pending_recv> pending;
	int next_req;
	int next_comm;
	state() : next_req(1), next_comm(16) {}
};

inline state& st() {
	static state s;
	return s;
}

/* Deliver a message into a pending receive if one matches; returns true if
 * it was delivered. */
inline bool deliver(const void *buf,size_t bytes,int tag,MPI_Comm comm) {
	state &s=st();
	for(std::list<pending_recv>::iterator it=s.pending.begin();it!=s.pending.end();++it) {
		if(it->tag==tag&&it->comm==comm) {
			if(bytes>it->cap) {
				fprintf(stderr,"mpi shim: message truncated (tag %d)\n",tag);
				abort();
			}
			memcpy(it->buf,buf,bytes);
			s.pending.erase(it);
			return true;
		}
	}
	return false;
}

inline bool is_pending(int id) {
	state &s=st();
	for(std::list<pending_recv>::iterator it=s.pending.begin();it!=s.pending.end();++it)
		if(it->id==id) return true;
	return false;
}

} // namespace pgmg_mpi_shim

inline int MPI_Init(int*,char***) {return MPI_SUCCESS;}
inline int MPI_Finalize() {return MPI_SUCCESS;}
inline int MPI_Barrier(MPI_Comm) {return MPI_SUCCESS;}
inline double MPI_Wtime() {
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC,&ts);
	return ts.tv_sec+1e-9*ts.tv_nsec;
}
inline int MPI_Abort(MPI_Comm,int code) {
	fprintf(stderr,"mpi shim: MPI_Abort(%d)\n",code);
	exit(code==0?1:code);
	return code;
}
inline int MPI_Comm_size(MPI_Comm,int *size) {*size=1;return MPI_SUCCESS;}
inline int MPI_Comm_rank(MPI_Comm,int *rank) {*rank=0;return MPI_SUCCESS;}
inline int MPI_Comm_dup(MPI_Comm,MPI_Comm *nc) {*nc=pgmg_mpi_shim::st().next_comm++;return MPI_SUCCESS;}
inline int MPI_Comm_free(MPI_Comm *c) {*c=MPI_COMM_NULL;return MPI_SUCCESS;}
inline int MPI_Comm_split(MPI_Comm,int color,int,MPI_Comm *nc) {
	*nc=color==MPI_UNDEFINED?MPI_COMM_NULL:pgmg_mpi_shim::st().next_comm++;
	return MPI_SUCCESS;
}
inline int MPI_Cart_create(MPI_Comm,int ndims,const int *dims,const int*,int,MPI_Comm *cart) {
	for(int i=0;i<ndims;i++) if(dims[i]!=1) {
		fprintf(stderr,"mpi shim: Cartesian grid must be 1x1x1 on one rank\n");
		abort();
	}
	*cart=pgmg_mpi_shim::st().next_comm++;
	return MPI_SUCCESS;
}
inline int MPI_Cart_coords(MPI_Comm,int,int maxdims,int *coords) {
	for(int i=0;i<maxdims;i++) coords[i]=0;
	return MPI_SUCCESS;
}
inline int MPI_Cart_rank(MPI_Comm,const int*,int *rank) {*rank=0;return MPI_SUCCESS;}

inline int MPI_Isend(const void *buf,int count,MPI_Datatype t,int,int tag,MPI_Comm comm,MPI_Request *req) {
	size_t bytes=count*pgmg_mpi_shim::type_size(t);
	if(!pgmg_mpi_shim::deliver(buf,bytes,tag,comm)) {
		pgmg_mpi_shim::message msg;
		msg.tag=tag;msg.comm=comm;
		msg.payload.assign(static_cast<const char*>(buf),static_cast<const char*>(buf)+bytes);
		pgmg_mpi_shim::st().queue.push_back(msg);
	}
	*req=0;
	return MPI_SUCCESS;
}
inline int MPI_Send(const void *buf,int count,MPI_Datatype t,int dest,int tag,MPI_Comm comm) {
	MPI_Request r;
	return MPI_Isend(buf,count,t,dest,tag,comm,&r);
}
inline int MPI_Irecv(void *buf,int count,MPI_Datatype t,int,int tag,MPI_Comm comm,MPI_Request *req) {
	pgmg_mpi_shim::state &s=pgmg_mpi_shim::st();
	size_t cap=count*pgmg_mpi_shim::type_size(t);
	for(std::list<pgmg_mpi_shim::message>::iterator it=s.queue.begin();it!=s.queue.end();++it) {
		if(it->tag==tag&&it->comm==comm) {
			if(it->payload.size()>cap) {
				fprintf(stderr,"mpi shim: message truncated (tag %d)\n",tag);
				abort();
			}
			if(!it->payload.empty()) memcpy(buf,&(it->payload[0]),it->payload.size());
			s.queue.erase(it);
			*req=0;
			return MPI_SUCCESS;
		}
	}
	pgmg_mpi_shim::pending_recv p;
	p.id=s.next_req++;p.tag=tag;p.comm=comm;p.buf=buf;p.cap=cap;
	s.pending.push_back(p);
	*req=p.id;
	return MPI_SUCCESS;
}
inline int MPI_Recv(void *buf,int count,MPI_Datatype t,int src,int tag,MPI_Comm comm,MPI_Status*) {
	MPI_Request r;
	MPI_Irecv(buf,count,t,src,tag,comm,&r);
	if(r!=0&&pgmg_mpi_shim::is_pending(r)) {
		fprintf(stderr,"mpi shim: blocking receive with no matching send (tag %d)\n",tag);
		abort();
	}
	return MPI_SUCCESS;
}
inline int MPI_Wait(MPI_Request *req,MPI_Status*) {
	if(*req!=0&&pgmg_mpi_shim::is_pending(*req)) {
		fprintf(stderr,"mpi shim: wait on a receive with no matching send\n");
		abort();
	}
	return MPI_SUCCESS;
}
inline int MPI_Waitall(int count,MPI_Request *reqs,MPI_Status*) {
	for(int i=0;i<count;i++) MPI_Wait(reqs+i,0);
	return MPI_SUCCESS;
}
inline int MPI_Allreduce(const void *in,void *out,int count,MPI_Datatype t,MPI_Op,MPI_Comm) {
	memmove(out,in,count*pgmg_mpi_shim::type_size(t));
	return MPI_SUCCESS;
}
inline int MPI_Reduce(const void *in,void *out,int count,MPI_Datatype t,MPI_Op,int,MPI_Comm) {
	memmove(out,in,count*pgmg_mpi_shim::type_size(t));
	return MPI_SUCCESS;
}
inline int MPI_Bcast(void*,int,MPI_Datatype,int,MPI_Comm) {return MPI_SUCCESS;}

#endif
